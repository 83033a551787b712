// Tile compositing, forward and backward
// (antialias/cuda_rasterizer/forward.cu:406-567, backward.cu:399-557).
//
// One CTA per 16x16 tile.  The tile's sorted pairs are contiguous 48-byte
// records (written by the last sort pass), so each 256-record batch is ONE
// bulk copy (cp.async.bulk, the TMA engine's 1-D form) into shared memory,
// completed on an mbarrier.  Three record buffers keep two batches in flight
// while the current one is composited.  A thread owns PPT pixels of one
// column (16 x 2*PPT pixels per warp); a warp whose pixels have all
// saturated (T < 1e-4) stops evaluating and only joins the per-batch barrier.
//
// Per-Gaussian outputs that the reference updates from every pixel (the
// racy out_point_weight max, the KPC statistics, the backward's 9 gradient
// atomics) are reduced across the warp first, then across the CTA in shared
// memory, and leave the CTA once per (tile, pair).
#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr int kBufs = 3;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false (and an error bit) if the copy never lands.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* err)
{
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > kSpinLimit) {
            set_error(err, FGS_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}
// 1-D bulk copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Issue the bulk copy of records [first, first+count) into buffer `buf`.
__device__ __forceinline__ void issue_batch(PairRecord* sbuf, uint64_t* bar, const PairRecord* recs, uint32_t first,
                                            uint32_t count)
{
    const uint32_t bytes = count * (uint32_t)sizeof(PairRecord);
    mbar_expect_tx(bar, bytes);
    bulk_g2s(sbuf, recs + first, bytes, bar);
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Conservative test used to skip (warp, record) pairs: can a Gaussian with mean
// (mx, my), conic (a, b, c) and opacity o reach alpha >= 1/255 at any pixel
// centre of [x0,x1] x [y0,y1]?  alpha <= o (power <= 0), so o < 1/255 never
// contributes; otherwise alpha >= 1/255 needs Q = a dx^2 + 2b dx dy + c dy^2
// <= 2 ln(255 o), and Q's minimum over the rectangle is 0 when the mean is
// inside, else on the boundary (one clamped 1-D minimum per edge).  The margin
// covers float rounding of the per-pixel evaluation by a wide factor; a
// non-positive-definite conic is never skipped.  Skipping only removes work
// that the per-pixel tests would reject, so every output is unchanged.
__device__ __forceinline__ bool may_touch(float mx, float my, float a, float b, float c, float o, float x0, float x1,
                                          float y0, float y1)
{
    if (!(o >= 1.0f / 255.0f)) return false;
    if (!(a > 0.f && c > 0.f && a * c - b * b > 0.f)) return true;
    const float X0 = x0 - mx, X1 = x1 - mx, Y0 = y0 - my, Y1 = y1 - my;
    if (X0 <= 0.f && X1 >= 0.f && Y0 <= 0.f && Y1 >= 0.f) return true;
    const float thr = 2.f * __logf(255.f * o);
    float q = 3.4e38f;
    // edges x = X0, X1
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const float X = i ? X1 : X0;
        const float dy = fminf(fmaxf(-b * X / c, Y0), Y1);
        q = fminf(q, a * X * X + 2.f * b * X * dy + c * dy * dy);
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const float Y = i ? Y1 : Y0;
        const float dx = fminf(fmaxf(-b * Y / a, X0), X1);
        q = fminf(q, a * dx * dx + 2.f * b * dx * Y + c * Y * Y);
    }
    const float mX = fmaxf(fabsf(X0), fabsf(X1)), mY = fmaxf(fabsf(Y0), fabsf(Y1));
    const float mag = a * mX * mX + c * mY * mY + 2.f * fabsf(b) * mX * mY;
    return q <= thr + 0.05f + 1e-5f * mag;
}

// ---------------------------------------------------------------- per-view render descriptors
// Everything one tile needs, for the plain launch (one view, one tile per CTA)
// and the persistent multi-view launch (CTAs pop (view, tile) work items).

template <int kBatch>
struct FwdSmem {
    PairRecord rec[kBufs][kBatch];
    uint64_t bar[kBufs];
    uint32_t wmax[2][kBatch];
    float ksum[2][kBatch];
    uint32_t kcnt[2][kBatch];
};

// Per-record gradient sums of a batch: warps 2s and 2s+1 add their warp totals
// into slot s.  A slot starts at zero and takes at most two additions, and
// float addition is commutative, so its value does not depend on which warp
// came first; the slots are then summed in slot order.  The result is the same
// on every run (no order-dependent float atomics anywhere in the backward).
template <int PPT>
constexpr int bwd_slots() { return (256 / PPT / 32) / 2 > 0 ? (256 / PPT / 32) / 2 : 1; }

template <int kBatch, int kSlots>
struct BwdSmem {
    PairRecord rec[kBufs][kBatch];
    uint64_t bar[kBufs];
    float acc[kSlots][9][kBatch];
    uint32_t max_last;
};

// ---------------------------------------------------------------- forward
// One tile.  Callers guarantee every thread of the CTA is synchronised on
// entry and that no bulk copy is in flight.  `gb` counts the record batches
// this CTA has ever waited for: batch g lives in buffer g % 3 and completes
// phase (g / 3) & 1 of that buffer's mbarrier, so the barriers are initialised
// once per CTA and keep their phase across tiles.
template <int PPT, int kBatch>
__device__ __forceinline__ void render_fwd_tile(FwdSmem<kBatch>& sm, const TileArgs& a, int tile, uint32_t& gb,
                                                unsigned* err)
{
    constexpr int NT = 256 / PPT;
    const int tid = threadIdx.x;
    const int W = a.W, H = a.H;
    const int gx = (W + kTileX - 1) / kTileX;
    const int bx = tile % gx, by = tile / gx;
    const int lx = tid & 15, ly0 = (tid >> 4) * PPT;
    const int px = bx * kTileX + lx;
    const uint2 range = a.ranges[tile];
    const uint32_t n = range.y - range.x;
    const int nb = (int)((n + kBatch - 1) / kBatch);
    const bool stats = a.kv_sum != nullptr;
    const PairRecord* recs = a.recs;

    if (tid == 0) {
        for (int b = 0; b < 2 && b < nb; b++) {
            const int buf = (int)((gb + b) % kBufs);
            issue_batch(sm.rec[buf], &sm.bar[buf], recs, range.x + b * kBatch, min((uint32_t)kBatch, n - b * kBatch));
        }
    }

    float T[PPT], C[PPT][3], wmax[PPT];
    uint32_t last[PPT];
    int maxid[PPT];
    bool done[PPT];
    float pyf[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
        T[k] = 1.0f;
        C[k][0] = C[k][1] = C[k][2] = 0.f;
        wmax[k] = 0.f;
        last[k] = 0;
        maxid[k] = -1;
        const int py = by * kTileY + ly0 + k;
        done[k] = !(px < W && py < H);
        pyf[k] = (float)py;
    }
    const float pxf = (float)px;
    // this warp's pixel rectangle: 16 columns x 2*PPT rows
    const float rx0 = (float)(bx * kTileX), rx1 = rx0 + (kTileX - 1);
    const float ry0 = (float)(by * kTileY + (tid >> 5) * 2 * PPT), ry1 = ry0 + (2 * PPT - 1);
    bool all_done = true;
#pragma unroll
    for (int k = 0; k < PPT; k++) all_done = all_done && done[k];

    int issued = nb < 2 ? nb : 2;
    uint32_t contributor = 0;
    for (int b = 0; b < nb; b++) {
        const uint32_t g = gb + b;
        const int buf = (int)(g % kBufs);
        const int acc = b & 1;
        const uint32_t cnt = min((uint32_t)kBatch, n - b * kBatch);
        if (!mbar_wait(&sm.bar[buf], (g / kBufs) & 1, err)) all_done = true;
        const PairRecord* R = sm.rec[buf];
        const bool warp_live = !__all_sync(0xffffffffu, all_done);
        if (warp_live) {
            bool stop = false;
            for (uint32_t k0 = 0; k0 < cnt && !stop; k0 += 32) {
                // which of these 32 records can reach alpha >= 1/255 inside this warp's pixels
                const uint32_t e = k0 + (tid & 31);
                bool t = false;
                if (e < cnt) {
                    const float4 ea = R[e].a, eb = R[e].b;
                    t = may_touch(ea.x, ea.y, ea.z, ea.w, eb.x, eb.y, rx0, rx1, ry0, ry1);
                }
                uint32_t live = __ballot_sync(0xffffffffu, t);
                while (live) {
                    const uint32_t j = k0 + (uint32_t)(__ffs(live) - 1);
                    live &= live - 1;
                    const uint32_t position = contributor + j + 1;
                    const float4 ra = R[j].a;
                    const float4 rb = R[j].b;
                    float wj = 0.f, ksum = 0.f;
                    uint32_t kc = 0;
#pragma unroll
                    for (int k = 0; k < PPT; k++) {
                        if (done[k]) continue;
                        const float2 d = {ra.x - pxf, ra.y - pyf[k]};
                        const float power = -0.5f * (ra.z * d.x * d.x + rb.x * d.y * d.y) - ra.w * d.x * d.y;
                        if (power > 0.0f) continue;
                        const float alpha = min(0.99f, rb.y * exp(power));
                        if (alpha < 1.0f / 255.0f) continue;
                        const float test_T = T[k] * (1 - alpha);
                        if (test_T < 0.0001f) {
                            done[k] = true;
                            continue;
                        }
                        const float4 rc = R[j].c;
                        C[k][0] += rb.z * alpha * T[k];
                        C[k][1] += rb.w * alpha * T[k];
                        C[k][2] += rc.x * alpha * T[k];
                        const float w = T[k] * alpha;
                        if (w > wmax[k]) {
                            wmax[k] = w;
                            maxid[k] = __float_as_int(rc.y);
                        }
                        wj = fmaxf(wj, w);
                        ksum += w;
                        kc += 1;
                        T[k] = test_T;
                        last[k] = position;
                    }
                    bool ad = true;
#pragma unroll
                    for (int k = 0; k < PPT; k++) ad = ad && done[k];
                    all_done = ad;
                    // per-Gaussian max weight (and statistics): warp, then CTA
                    if (__any_sync(0xffffffffu, wj > 0.f)) {
                        const uint32_t wm = __reduce_max_sync(0xffffffffu, __float_as_uint(wj));
                        float ks = 0.f;
                        uint32_t kcs = 0;
                        if (stats) {
                            ks = warp_sum(ksum);
                            kcs = __reduce_add_sync(0xffffffffu, kc);
                        }
                        if ((tid & 31) == 0) {
                            atomicMax(&sm.wmax[acc][j], wm);
                            if (stats) {
                                atomicAdd(&sm.ksum[acc][j], ks);
                                atomicAdd(&sm.kcnt[acc][j], kcs);
                            }
                        }
                    }
                    if (__all_sync(0xffffffffu, all_done)) {
                        stop = true;
                        break;
                    }
                }
            }
        }
        contributor += cnt;
        const int ndone = __syncthreads_count(all_done);
        for (uint32_t e = tid; e < cnt; e += NT) {
            const uint32_t wm = sm.wmax[acc][e];
            if (wm) {
                const int id = __float_as_int(R[e].c.y);
                if (a.out_point_weight) atomicMax(reinterpret_cast<unsigned*>(a.out_point_weight) + id, wm);
                sm.wmax[acc][e] = 0;
            }
            if (stats) {
                a.kv_sum[range.x + b * kBatch + e] = sm.ksum[acc][e];
                a.kv_cnt[range.x + b * kBatch + e] = sm.kcnt[acc][e];
                sm.ksum[acc][e] = 0.f;
                sm.kcnt[acc][e] = 0;
            }
        }
        if (ndone == NT) {
            // drain the copy still in flight before the buffers are reused or the CTA exits
            if (tid == 0 && b + 1 < nb)
                mbar_wait(&sm.bar[(g + 1) % kBufs], ((g + 1) / kBufs) & 1, err);
            if (stats) {
                // pairs never reached contribute nothing
                for (uint32_t e = (b + 1) * kBatch + tid; e < n; e += NT) {
                    a.kv_sum[range.x + e] = 0.f;
                    a.kv_cnt[range.x + e] = 0;
                }
            }
            break;
        }
        if (b + 2 < nb) {
            if (tid == 0) {
                const int nbuf = (int)((g + 2) % kBufs);
                issue_batch(sm.rec[nbuf], &sm.bar[nbuf], recs, range.x + (b + 2) * kBatch,
                            min((uint32_t)kBatch, n - (b + 2) * kBatch));
            }
            issued = b + 3;
        }
    }
    gb += (uint32_t)issued;

#pragma unroll
    for (int k = 0; k < PPT; k++) {
        const int py = by * kTileY + ly0 + k;
        if (px < W && py < H) {
            const int pix = W * py + px;
            a.final_T[pix] = T[k];
            a.n_contrib[pix] = last[k];
            a.out_color[pix] = C[k][0] + T[k] * a.bg[0];
            a.out_color[H * W + pix] = C[k][1] + T[k] * a.bg[1];
            a.out_color[2 * H * W + pix] = C[k][2] + T[k] * a.bg[2];
            if (a.out_point_id) a.out_point_id[pix] = maxid[k];
            if (a.out_pw_pixel) a.out_pw_pixel[pix] = wmax[k];
        }
    }
}

template <int kBatch>
__device__ __forceinline__ void fwd_smem_init(FwdSmem<kBatch>& sm, int NT)
{
    for (int e = threadIdx.x; e < 2 * kBatch; e += NT) {
        (&sm.wmax[0][0])[e] = 0;
        (&sm.ksum[0][0])[e] = 0.f;
        (&sm.kcnt[0][0])[e] = 0;
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kBufs; i++) mbar_init(&sm.bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
}

template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT) render_fwd_kernel(TileArgs a, unsigned* err)
{
    __shared__ __align__(128) FwdSmem<kBatch> sm;
    fwd_smem_init(sm, 256 / PPT);
    uint32_t gb = 0;
    render_fwd_tile<PPT, kBatch>(sm, a, blockIdx.x, gb, err);
}

// Persistent multi-view forward: CTAs pop work items from one queue; item i is
// tile (i - begin[v]) of view v.  Views are laid out in the caller's order.
template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT)
    render_fwd_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin, int nviews,
                            uint32_t total, uint32_t* queue, unsigned* err)
{
    __shared__ __align__(128) FwdSmem<kBatch> sm;
    __shared__ uint32_t s_item;
    fwd_smem_init(sm, 256 / PPT);
    uint32_t gb = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total) break;
        int v = 0;
        while (v + 1 < nviews && begin[v + 1] <= item) v++;
        const TileArgs a = views[v];
        render_fwd_tile<PPT, kBatch>(sm, a, (int)(item - begin[v]), gb, err);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- backward
template <int PPT, int kBatch>
__device__ __forceinline__ void render_bwd_tile(BwdSmem<kBatch, bwd_slots<PPT>()>& sm, const TileArgs& a, int tile,
                                                uint32_t& gb, int consistent, unsigned* err)
{
    constexpr int kSlots = bwd_slots<PPT>();
    constexpr int NT = 256 / PPT;
    constexpr int NG = 9;  // dcolor r,g,b ; dmean2D x,y ; dconic x,y,w ; dopacity
    const int tid = threadIdx.x;
    const int W = a.W, H = a.H;
    const int gx = (W + kTileX - 1) / kTileX;
    const int bx = tile % gx, by = tile / gx;
    const int lx = tid & 15, ly0 = (tid >> 4) * PPT;
    const int px = bx * kTileX + lx;
    const uint2 range = a.ranges[tile];
    const PairRecord* recs = a.recs;

    float T[PPT], T_final[PPT], dpix[PPT][3], accum[PPT][3], last_color[PPT][3], last_alpha[PPT], pyf[PPT];
    uint32_t last[PPT];
    float bg_dot[PPT];
    const float bg0 = a.bg[0], bg1 = a.bg[1], bg2 = a.bg[2];
    uint32_t my_max = 0;
#pragma unroll
    for (int k = 0; k < PPT; k++) {
        const int py = by * kTileY + ly0 + k;
        const bool inside = px < W && py < H;
        const int pix = W * py + px;
        T_final[k] = inside ? a.final_T[pix] : 0.f;
        T[k] = T_final[k];
        last[k] = inside ? a.n_contrib[pix] : 0;
        my_max = max(my_max, last[k]);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dpix[k][c] = inside ? a.dL_dpix[c * H * W + pix] : 0.f;
            accum[k][c] = 0.f;
            last_color[k][c] = 0.f;
        }
        last_alpha[k] = 0.f;
        bg_dot[k] = bg0 * dpix[k][0] + bg1 * dpix[k][1] + bg2 * dpix[k][2];
        pyf[k] = (float)py;
    }
    const float pxf = (float)px;
    const float rx0 = (float)(bx * kTileX), rx1 = rx0 + (kTileX - 1);
    const float ry0 = (float)(by * kTileY + (tid >> 5) * 2 * PPT), ry1 = ry0 + (2 * PPT - 1);
    const float ddelx_dx = 0.5 * W;
    const float ddely_dy = 0.5 * H;

    if (tid == 0) sm.max_last = 0;
    __syncthreads();
    const uint32_t warp_last = __reduce_max_sync(0xffffffffu, my_max);
    if ((tid & 31) == 0) atomicMax(&sm.max_last, warp_last);
    __syncthreads();
    // Entries at or beyond the largest n_contrib of the tile touch no pixel.
    const uint32_t n = min(range.y - range.x, sm.max_last);
    const int nb = (int)((n + kBatch - 1) / kBatch);
    // batch b holds entries [lo_b, hi_b) with hi_b = n - b*kBatch (back to front)
    if (tid == 0) {
        for (int b = 0; b < 2 && b < nb; b++) {
            const uint32_t hi = n - b * kBatch, lo = hi > (uint32_t)kBatch ? hi - kBatch : 0;
            const int buf = (int)((gb + b) % kBufs);
            issue_batch(sm.rec[buf], &sm.bar[buf], recs, range.x + lo, hi - lo);
        }
    }

    for (int b = 0; b < nb; b++) {
        const uint32_t g = gb + b;
        const int buf = (int)(g % kBufs);
        const uint32_t hi = n - b * kBatch, lo = hi > (uint32_t)kBatch ? hi - kBatch : 0;
        const uint32_t cnt = hi - lo;
        mbar_wait(&sm.bar[buf], (g / kBufs) & 1, err);
        const PairRecord* R = sm.rec[buf];
        for (int k0 = (int)((cnt - 1) & ~31u); k0 >= 0; k0 -= 32) {
            // records of this chunk that sit before some pixel's last contributor and can
            // reach alpha >= 1/255 inside this warp's pixels, walked back to front
            const uint32_t e = (uint32_t)k0 + (tid & 31);
            bool t = false;
            if (e < cnt && lo + e < warp_last) {
                const float4 ea = R[e].a, eb = R[e].b;
                t = may_touch(ea.x, ea.y, ea.z, ea.w, eb.x, eb.y, rx0, rx1, ry0, ry1);
            }
            uint32_t live = __ballot_sync(0xffffffffu, t);
            while (live) {
                const int bit = 31 - __clz(live);
                live &= ~(1u << bit);
                const int j = k0 + bit;
                const uint32_t contributor = lo + (uint32_t)j;  // 0-based position in the tile list
                const float4 ra = R[j].a;
                const float4 rb = R[j].b;
                float gr[NG];
#pragma unroll
                for (int q = 0; q < NG; q++) gr[q] = 0.f;
                bool any = false;
#pragma unroll
                for (int k = 0; k < PPT; k++) {
                    if (contributor >= last[k]) continue;
                    const float2 d = {ra.x - pxf, ra.y - pyf[k]};
                    const float power = -0.5f * (ra.z * d.x * d.x + rb.x * d.y * d.y) - ra.w * d.x * d.y;
                    if (power > 0.0f) continue;
                    const float G = exp(power);
                    const float alpha = min(0.99f, rb.y * G);
                    if (alpha < 1.0f / 255.0f) continue;
                    // transmittance before this Gaussian (fast reciprocal: 1 - alpha >= 0.01)
                    const float inv_1ma = __fdividef(1.f, 1.f - alpha);
                    T[k] = T[k] * inv_1ma;
                    const float dchannel_dcolor = alpha * T[k];
                    const float col[3] = {rb.z, rb.w, R[j].c.x};
                    float dL_dalpha = 0.0f;
#pragma unroll
                    for (int ch = 0; ch < 3; ch++) {
                        const float c = col[ch];
                        accum[k][ch] = last_alpha[k] * last_color[k][ch] + (1.f - last_alpha[k]) * accum[k][ch];
                        last_color[k][ch] = c;
                        dL_dalpha += (c - accum[k][ch]) * dpix[k][ch];
                        gr[ch] += dchannel_dcolor * dpix[k][ch];
                    }
                    dL_dalpha *= T[k];
                    last_alpha[k] = alpha;
                    // background term; exactly zero (and skipped) for a black background
                    if (bg_dot[k] != 0.f) dL_dalpha += (-T_final[k] * inv_1ma) * bg_dot[k];
                    if (consistent && rb.y * G > 0.99f) dL_dalpha = 0.f;
                    const float dL_dG = rb.y * dL_dalpha;
                    const float gdx = G * d.x;
                    const float gdy = G * d.y;
                    const float dG_ddelx = -gdx * ra.z - gdy * ra.w;
                    const float dG_ddely = -gdy * rb.x - gdx * ra.w;
                    gr[3] += dL_dG * dG_ddelx * ddelx_dx;
                    gr[4] += dL_dG * dG_ddely * ddely_dy;
                    gr[5] += -0.5f * gdx * d.x * dL_dG;
                    gr[6] += -0.5f * gdx * d.y * dL_dG;
                    gr[7] += -0.5f * gdy * d.y * dL_dG;
                    gr[8] += G * dL_dalpha;
                    any = true;
                }
                if (__any_sync(0xffffffffu, any)) {
                    const float tot = warp_transpose_sum9(gr);
                    const unsigned lane = tid & 31;
                    if (!(lane & 1) && (lane >> 1) < NG) atomicAdd(&sm.acc[(tid >> 5) >> 1][lane >> 1][j], tot);
                }
            }
        }
        __syncthreads();
        // this batch's per-pair gradients, at each pair's emission index
        for (uint32_t e = tid; e < cnt; e += NT) {
            float* dst = a.pgrad + (size_t)__float_as_uint(R[e].c.w) * NG;
#pragma unroll
            for (int q = 0; q < NG; q++) {
                float v = 0.f;
#pragma unroll
                for (int sl = 0; sl < kSlots; sl++) {
                    v += sm.acc[sl][q][e];
                    sm.acc[sl][q][e] = 0.f;
                }
                dst[q] = v;
            }
        }
        if (tid == 0 && b + 2 < nb) {
            const int nbuf = (int)((g + 2) % kBufs);
            const uint32_t hi2 = n - (b + 2) * kBatch, lo2 = hi2 > (uint32_t)kBatch ? hi2 - kBatch : 0;
            issue_batch(sm.rec[nbuf], &sm.bar[nbuf], recs, range.x + lo2, hi2 - lo2);
        }
        __syncthreads();
    }
    gb += (uint32_t)nb;
    // pairs at or past the tile's largest n_contrib touch no pixel: zero gradients
    for (uint32_t e = n + tid; e < range.y - range.x; e += NT) {
        float* dst = a.pgrad + (size_t)__float_as_uint(recs[range.x + e].c.w) * NG;
#pragma unroll
        for (int q = 0; q < NG; q++) dst[q] = 0.f;
    }
}

template <int kBatch, int kSlots>
__device__ __forceinline__ void bwd_smem_init(BwdSmem<kBatch, kSlots>& sm, int NT)
{
    for (int e = threadIdx.x; e < kSlots * 9 * kBatch; e += NT) (&sm.acc[0][0][0])[e] = 0.f;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kBufs; i++) mbar_init(&sm.bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
}

// The backward's shared state can pass the 48 KB static limit (8 warps, 256-record
// batches): it lives in dynamic shared memory.
template <int PPT, int kBatch>
using BwdSmemT = BwdSmem<kBatch, bwd_slots<PPT>()>;

template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT) render_bwd_kernel(TileArgs a, int consistent, unsigned* err)
{
    extern __shared__ __align__(128) unsigned char bwd_dyn[];
    BwdSmemT<PPT, kBatch>& sm = *reinterpret_cast<BwdSmemT<PPT, kBatch>*>(bwd_dyn);
    bwd_smem_init(sm, 256 / PPT);
    uint32_t gb = 0;
    render_bwd_tile<PPT, kBatch>(sm, a, blockIdx.x, gb, consistent, err);
}

template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT)
    render_bwd_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin, int nviews,
                            uint32_t total, uint32_t* queue, int consistent, unsigned* err)
{
    extern __shared__ __align__(128) unsigned char bwd_dyn[];
    BwdSmemT<PPT, kBatch>& sm = *reinterpret_cast<BwdSmemT<PPT, kBatch>*>(bwd_dyn);
    __shared__ uint32_t s_item;
    bwd_smem_init(sm, 256 / PPT);
    uint32_t gb = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total) break;
        int v = 0;
        while (v + 1 < nviews && begin[v + 1] <= item) v++;
        const TileArgs a = views[v];
        render_bwd_tile<PPT, kBatch>(sm, a, (int)(item - begin[v]), gb, consistent, err);
        __syncthreads();
    }
}

}  // namespace

namespace {
RenderConfig g_cfg{2, 256, 2, 256};

template <int PPT, int B>
void fwd_launch(int grid, const ImageState& im, const BinState& b, int W, int H, const float* bg, float* out_color,
                int* point_id, float* pw_pixel, float* point_weight, bool stats, unsigned* err, cudaStream_t s)
{
    TileArgs a{};
    a.ranges = im.ranges; a.recs = b.rec; a.W = W; a.H = H; a.bg = bg;
    a.out_color = out_color; a.final_T = im.final_T; a.n_contrib = im.n_contrib; a.out_point_id = point_id;
    a.out_pw_pixel = pw_pixel; a.out_point_weight = point_weight;
    a.kv_sum = stats ? b.kv_sum : nullptr; a.kv_cnt = stats ? b.kv_cnt : nullptr;
    render_fwd_kernel<PPT, B><<<grid, 256 / PPT, 0, s>>>(a, err);
}

// Dynamic shared memory of a backward kernel instantiation (opted in once per process
// and device ordinal; Tag tells the single-view and multi-view kernels apart).
template <int PPT, int B, int Tag, typename Kern>
size_t bwd_smem_bytes(Kern k)
{
    static bool done[64] = {};
    const size_t bytes = sizeof(BwdSmemT<PPT, B>);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !done[dev]) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (dev >= 0 && dev < 64) done[dev] = true;
    }
    return bytes;
}

template <int PPT, int B>
void bwd_launch(int grid, const ImageState& im, const BinState& b, int W, int H, const float* bg, const float* dL,
                int consistent, unsigned* err, cudaStream_t s)
{
    TileArgs a{};
    a.ranges = im.ranges; a.recs = b.rec; a.W = W; a.H = H; a.bg = bg;
    a.final_T = im.final_T; a.n_contrib = im.n_contrib;
    a.dL_dpix = dL; a.pgrad = b.pgrad;
    const size_t smem = bwd_smem_bytes<PPT, B, 0>(render_bwd_kernel<PPT, B>);
    render_bwd_kernel<PPT, B><<<grid, 256 / PPT, smem, s>>>(a, consistent, err);
}

#define FGS_RENDER_DISPATCH(FN, PPT_, B_, ...)                                            \
    do {                                                                                  \
        const int ppt_ = (PPT_), b_ = (B_);                                               \
        if (ppt_ == 1 && b_ == 64) FN<1, 64>(__VA_ARGS__);                                \
        else if (ppt_ == 1 && b_ == 128) FN<1, 128>(__VA_ARGS__);                         \
        else if (ppt_ == 1) FN<1, 256>(__VA_ARGS__);                                      \
        else if (ppt_ == 2 && b_ == 64) FN<2, 64>(__VA_ARGS__);                           \
        else if (ppt_ == 2 && b_ == 128) FN<2, 128>(__VA_ARGS__);                         \
        else if (ppt_ == 2) FN<2, 256>(__VA_ARGS__);                                      \
        else if (ppt_ == 4 && b_ == 64) FN<4, 64>(__VA_ARGS__);                           \
        else if (ppt_ == 4 && b_ == 128) FN<4, 128>(__VA_ARGS__);                         \
        else FN<4, 256>(__VA_ARGS__);                                                     \
    } while (0)
}  // namespace

bool valid_render_config(const RenderConfig& c)
{
    auto ok_p = [](int v) { return v == 1 || v == 2 || v == 4; };
    auto ok_b = [](int v) { return v == 64 || v == 128 || v == 256; };
    return ok_p(c.fwd_ppt) && ok_p(c.bwd_ppt) && ok_b(c.fwd_batch) && ok_b(c.bwd_batch);
}
void set_render_config(const RenderConfig& c) { g_cfg = c; }
RenderConfig get_render_config() { return g_cfg; }

void launch_render_fwd(int W, int H, const ImageState& im, const BinState& b, const float* bg, float* out_color,
                       int* point_id, float* pw_pixel, float* point_weight, bool stats, unsigned* err,
                       cudaStream_t s)
{
    const int gx = (W + kTileX - 1) / kTileX, gy = (H + kTileY - 1) / kTileY;
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(fwd_launch, c.fwd_ppt, c.fwd_batch, gx * gy, im, b, W, H, bg, out_color, point_id, pw_pixel,
                        point_weight, stats, err, s);
    note_launches(1);
}

namespace {
template <int PPT, int B>
void fwd_multi_launch(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total, uint32_t* queue,
                      unsigned* err, cudaStream_t s)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_fwd_multi_kernel<PPT, B>, 256 / PPT, 0);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    render_fwd_multi_kernel<PPT, B><<<grid, 256 / PPT, 0, s>>>(views, begin, nviews, total, queue, err);
}

template <int PPT, int B>
void bwd_multi_launch(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total, uint32_t* queue,
                      int consistent, unsigned* err, cudaStream_t s)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = bwd_smem_bytes<PPT, B, 1>(render_bwd_multi_kernel<PPT, B>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_bwd_multi_kernel<PPT, B>, 256 / PPT, smem);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    render_bwd_multi_kernel<PPT, B><<<grid, 256 / PPT, smem, s>>>(views, begin, nviews, total, queue, consistent,
                                                                  err);
}
}  // namespace

void launch_render_fwd_multi(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total_tiles,
                             uint32_t* queue, unsigned* err, cudaStream_t s)
{
    cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(fwd_multi_launch, c.fwd_ppt, c.fwd_batch, views, begin, nviews, total_tiles, queue, err, s);
    note_launches(1);
}

void launch_render_bwd_multi(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total_tiles,
                             uint32_t* queue, int consistent, unsigned* err, cudaStream_t s)
{
    cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(bwd_multi_launch, c.bwd_ppt, c.bwd_batch, views, begin, nviews, total_tiles, queue,
                        consistent, err, s);
    note_launches(1);
}

void launch_render_bwd(int W, int H, const ImageState& im, const BinState& b, const float* bg,
                       const float* dL_dpix, int consistent, unsigned* err, cudaStream_t s)
{
    const int gx = (W + kTileX - 1) / kTileX, gy = (H + kTileY - 1) / kTileY;
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(bwd_launch, c.bwd_ppt, c.bwd_batch, gx * gy, im, b, W, H, bg, dL_dpix, consistent, err, s);
    note_launches(1);
}

}  // namespace fgs
