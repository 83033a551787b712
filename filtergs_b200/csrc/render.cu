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
#include <cstddef>

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
    WaitBound wb;
    while (!mbar_try_wait(bar, parity)) {
        if (wb.expired(kWaitLimitNs)) {
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

// The statistics sums come last: a launch without statistics allocates the
// dynamic shared memory only up to ksum (fwd_smem_bytes), which leaves room for
// one more CTA per SM at the batch sizes the autotuner picks.
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
// One (pixel, record) step of the compositing loop (forward.cu:466-544), in two
// parts.  fwd_alpha: the Gaussian's alpha at the pixel centre, or 0 where the
// reference skips the record (power > 0, alpha < 1/255); it does not depend on
// the pixel's state, so a renderer may evaluate several records ahead.
// fwd_accumulate: early termination below T = 1e-4, the colour and
// transmittance update and the pixel's strongest contributor; returns the
// weight T * alpha the record took (> 0), or 0 when it did not contribute.
//
// The multiply-adds are spelled out with round-to-nearest intrinsics (the
// contraction a compiler would pick for the reference's expressions), so that
// the compiler cannot fuse them differently in different renderers: the tile
// path at any pixels-per-thread and the band path produce the same bits.
__device__ __forceinline__ float fwd_alpha(const float4 ra, const float4 rb, float pxf, float pyf)
{
    const float dx = ra.x - pxf, dy = ra.y - pyf;
    // -0.5 * (a dx^2 + c dy^2) - b dx dy with the first product of each sum fused
    // into the multiply-add: of the orders measured, the one whose alphas agree
    // with the reference build's on the most pixels
    const float q = __fmaf_rn(__fmul_rn(ra.z, dx), dx, __fmul_rn(__fmul_rn(rb.x, dy), dy));
    const float power = __fmaf_rn(-0.5f, q, -__fmul_rn(__fmul_rn(ra.w, dx), dy));
    if (power > 0.0f) return 0.f;
    const float alpha = fminf(0.99f, __fmul_rn(rb.y, expf(power)));
    return alpha < 1.0f / 255.0f ? 0.f : alpha;
}

__device__ __forceinline__ float fwd_accumulate(float alpha, const float4 rb, const PairRecord& rec,
                                                uint32_t position, float& T, float (&C)[3], float& wmax, int& maxid,
                                                uint32_t& last, bool& done)
{
    if (done || alpha == 0.f) return 0.f;
    const float test_T = __fmul_rn(T, 1.0f - alpha);
    if (test_T < 0.0001f) {
        done = true;
        return 0.f;
    }
    const float4 rc = rec.c;
    C[0] = __fmaf_rn(__fmul_rn(rb.z, alpha), T, C[0]);
    C[1] = __fmaf_rn(__fmul_rn(rb.w, alpha), T, C[1]);
    C[2] = __fmaf_rn(__fmul_rn(rc.x, alpha), T, C[2]);
    const float w = __fmul_rn(T, alpha);
    if (w > wmax) {
        wmax = w;
        maxid = __float_as_int(rc.y);
    }
    T = test_T;
    last = position;
    return w;
}

// fwd_alpha + fwd_accumulate in one pass with early exits (the tile path: no
// record is evaluated ahead), the same arithmetic.  A contribution also goes into
// the caller's per-record sums (max weight, weight sum, count).
__device__ __forceinline__ void fwd_pixel_step(const float4 ra, const float4 rb, const PairRecord& rec, float pxf,
                                               float pyf, uint32_t position, float& T, float (&C)[3], float& wmax,
                                               int& maxid, uint32_t& last, bool& done, float& wj, float& ksum,
                                               uint32_t& kc)
{
    if (done) return;
    const float dx = ra.x - pxf, dy = ra.y - pyf;
    const float q = __fmaf_rn(__fmul_rn(ra.z, dx), dx, __fmul_rn(__fmul_rn(rb.x, dy), dy));
    const float power = __fmaf_rn(-0.5f, q, -__fmul_rn(__fmul_rn(ra.w, dx), dy));
    if (power > 0.0f) return;
    const float alpha = fminf(0.99f, __fmul_rn(rb.y, expf(power)));
    if (alpha < 1.0f / 255.0f) return;
    const float test_T = __fmul_rn(T, 1.0f - alpha);
    if (test_T < 0.0001f) {
        done = true;
        return;
    }
    const float4 rc = rec.c;
    C[0] = __fmaf_rn(__fmul_rn(rb.z, alpha), T, C[0]);
    C[1] = __fmaf_rn(__fmul_rn(rb.w, alpha), T, C[1]);
    C[2] = __fmaf_rn(__fmul_rn(rc.x, alpha), T, C[2]);
    const float w = __fmul_rn(T, alpha);
    if (w > wmax) {
        wmax = w;
        maxid = __float_as_int(rc.y);
    }
    wj = fmaxf(wj, w);
    ksum += w;
    kc += 1;
    T = test_T;
    last = position;
}

// One tile.  Callers guarantee every thread of the CTA is synchronised on
// entry and that no bulk copy is in flight.  `gb` counts the record batches
// this CTA has ever waited for: batch g lives in buffer g % 3 and completes
// phase (g / 3) & 1 of that buffer's mbarrier, so the barriers are initialised
// once per CTA and keep their phase across tiles.
template <int PPT, int kBatch>
__device__ __forceinline__ void render_fwd_tile(FwdSmem<kBatch>& sm, const TileArgs& a, int tile, uint32_t& gb,
                                                uint32_t split_min, bool stats_smem, unsigned* err)
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
    if (split_min && n >= split_min) return;  // rendered in bands (render_long_tile)
    const int nb = (int)((n + kBatch - 1) / kBatch);
    const bool stats = stats_smem && a.kv_sum != nullptr;  // the sums exist only in a launch that has them
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
                    for (int k = 0; k < PPT; k++)
                        fwd_pixel_step(ra, rb, R[j], pxf, pyf[k], position, T[k], C[k], wmax[k], maxid[k], last[k],
                                       done[k], wj, ksum, kc);
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
            a.out_color[pix] = __fmaf_rn(T[k], a.bg[0], C[k][0]);
            a.out_color[H * W + pix] = __fmaf_rn(T[k], a.bg[1], C[k][1]);
            a.out_color[2 * H * W + pix] = __fmaf_rn(T[k], a.bg[2], C[k][2]);
            if (a.out_point_id) a.out_point_id[pix] = maxid[k];
            if (a.out_pw_pixel) a.out_pw_pixel[pix] = wmax[k];
        }
    }
}

template <int kBatch>
__device__ __forceinline__ void fwd_smem_init(FwdSmem<kBatch>& sm, int NT, bool stats_smem)
{
    for (int e = threadIdx.x; e < 2 * kBatch; e += NT) {
        (&sm.wmax[0][0])[e] = 0;
        if (stats_smem) {
            (&sm.ksum[0][0])[e] = 0.f;
            (&sm.kcnt[0][0])[e] = 0;
        }
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kBufs; i++) mbar_init(&sm.bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
}

// Resident CTAs per SM the forward kernels are compiled for (a register cap of
// 65536 / (CTAs x threads)): 32 warps per SM at 2 and at 4 pixels per thread (64
// registers, at 4 with a few spilled bytes; a 64- or 128-record batch's shared
// memory then lets them fill; measured faster than 24 and 28 warps without or with
// fewer spills).
template <int PPT>
constexpr int fwd_min_ctas() { return PPT == 1 ? 3 : (PPT == 2 ? 8 : 16); }

template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT, fwd_min_ctas<PPT>())
    render_fwd_kernel(TileArgs a, uint32_t split_min, unsigned* err)
{
    extern __shared__ __align__(128) unsigned char fwd_dyn[];
    FwdSmem<kBatch>& sm = *reinterpret_cast<FwdSmem<kBatch>*>(fwd_dyn);
    const bool stats_smem = a.kv_sum != nullptr;  // the launch sized the shared memory from the same test
    fwd_smem_init(sm, 256 / PPT, stats_smem);
    uint32_t gb = 0;
    render_fwd_tile<PPT, kBatch>(sm, a, blockIdx.x, gb, split_min, stats_smem, err);
}

// Persistent multi-view forward: CTAs pop work items from one queue; item i is
// tile (i - begin[v]) of view v.  Views are laid out in the caller's order.
__device__ __forceinline__ int view_of(const uint32_t* __restrict__ begin, int nviews, uint32_t item)
{
    int v = 0;
    while (v + 1 < nviews && begin[v + 1] <= item) v++;
    return v;
}

template <int PPT, int kBatch>
__global__ void __launch_bounds__(256 / PPT, fwd_min_ctas<PPT>())
    render_fwd_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin, int nviews,
                            uint32_t total, uint32_t* queue, uint32_t split_min, unsigned* err)
{
    // launched without the statistics sums (the batched path keeps no statistics)
    extern __shared__ __align__(128) unsigned char fwd_dyn[];
    FwdSmem<kBatch>& sm = *reinterpret_cast<FwdSmem<kBatch>*>(fwd_dyn);
    __shared__ uint32_t s_item;
    fwd_smem_init(sm, 256 / PPT, false);
    uint32_t gb = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total) break;
        const int v = view_of(begin, nviews, item);
        const TileArgs& a = views[v];  // fields read where used, not held in registers
        render_fwd_tile<PPT, kBatch>(sm, a, (int)(item - begin[v]), gb, split_min, false, err);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- long tiles in bands
// A tile with a long record list (dense small splats: distant LoD levels, a
// horizon) is the critical path of the one-CTA-per-tile render: its few warps
// walk every record while the rest of the GPU has finished.  Tiles with at
// least split_min records are rendered instead in bands of BW x BH pixels, one
// warp per band and four bands per CTA (a tile's 256 / (BW BH) bands spread over
// several SMs), longest tiles first.  The CTA stages the tile's records in
// chunks of two records per thread (plain coalesced loads; the next chunk is
// loaded into registers while the current one is composited), and each thread
// works out which bands its record can reach (band_mask), so a record is tested
// once per four bands instead of once per band, and a warp finds its band's
// records with one ballot per 32.  The
// warp composites them with the tile path's per-pixel functions; a band of
// fewer than 32 pixels evaluates several records per step (lane = slot * pixels
// + pixel) and the pixel's owner lane composites them in order.  Every pixel
// composites the same records in the same order with the same arithmetic as on
// the tile path.  Per record, a contributing lane folds its weight into the
// record's shared slot; the slots leave once per chunk (atomicMax into the
// per-Gaussian max weight, atomicAdd into the statistics, which are zeroed
// before the launch when on).
//
// Order: long tiles are binned by floor(log2(records)) (kLongBuckets bins of
// capacity `cap` each); the queue hands out the bins from the longest down.
constexpr int kLongBuckets = 32;

template <int BW, int BH>
struct LongTile {
    static_assert(BW * BH <= 32 && kTileX % BW == 0 && kTileY % BH == 0, "band shape");
    static constexpr int kPix = BW * BH;                   // pixels per band
    static constexpr int kPerRow = kTileX / BW;            // bands per row of the tile
    static constexpr int kRows = kTileY / BH;
    static constexpr int kBands = kPerRow * kRows;         // bands per tile
    static constexpr int kGroup = kBands < 4 ? kBands : 4; // bands (warps) per CTA
    static constexpr int kGroups = kBands / kGroup;        // CTAs per tile
    static constexpr int kThreads = 32 * kGroup;
    static constexpr int kPer = 2;                         // records each thread stages per chunk
    static constexpr int kChunk = kPer * kThreads;
    static constexpr int kSlots = 32 / kPix;               // records evaluated per step
};

template <int kChunk>
struct LongSmem {
    PairRecord rec[kChunk];
    uint32_t mask[kChunk];  // bands each record can reach
    uint32_t wmax[kChunk];  // per record: max weight over the tile's pixels
    float ksum[kChunk];     // statistics: weight sum and count over the tile's pixels
    uint32_t kcnt[kChunk];
};

// The bands of the tile at (tx0, ty0) that a record can reach.  The record
// reaches alpha >= 1/255 only inside the ellipse Q(d) = a dx^2 + 2 b dx dy +
// c dy^2 <= 2 ln(255 o); the test uses the axis-aligned box around Q(d) <= t,
// t = 1.01 * 2 ln(255 o) + 0.1, whose half-widths are sqrt(t c / det) and
// sqrt(t a / det) (det = a c - b^2), grown by 0.01 px.  With det >= 0.01 a c the
// per-pixel float evaluation of Q errs by under 5e-7 of a dx^2 + c dy^2 +
// 2|b dx dy|, which is at most 400 Q there, far inside the 1% margin; the fast
// log and divide err by less than the 0.1 absolute margin.  So a pixel outside
// the box gets alpha < 1/255 and is skipped by the per-pixel test anyway.  Band
// k of a row covers the pixel columns tx0 + k BW .. tx0 + k BW + BW - 1, so the
// box reaches it when mx - ex <= tx0 + k BW + BW - 1 and mx + ex >= tx0 + k BW
// (rows alike).  0 when the record cannot reach alpha >= 1/255 in the tile;
// every band for a conic the box does not cover (near-degenerate, not positive
// definite, not finite) and for a mean that is not finite.
template <int BW, int BH>
__device__ __forceinline__ uint32_t band_mask(const float4 ea, const float4 eb, float tx0, float ty0)
{
    using L = LongTile<BW, BH>;
    constexpr uint32_t kAll = L::kBands == 32 ? 0xffffffffu : ((1u << L::kBands) - 1u);
    const float mx = ea.x, my = ea.y, a = ea.z, b = ea.w, c = eb.x, o = eb.y;
    if (!(o >= 1.0f / 255.0f)) return 0u;
    const float det = a * c - b * b;
    if (!(a > 0.f && c > 0.f && det >= 0.01f * a * c) || !isfinite(mx) || !isfinite(my)) return kAll;
    const float t = 1.01f * (2.f * __logf(255.f * o)) + 0.1f;
    const float s = __fdividef(t, det);
    const float ex = sqrtf(s * c) + 0.01f, ey = sqrtf(s * a) + 0.01f;
    const float lo_x = (mx - ex - tx0 - (BW - 1)) * (1.f / BW), hi_x = (mx + ex - tx0) * (1.f / BW);
    const float lo_y = (my - ey - ty0 - (BH - 1)) * (1.f / BH), hi_y = (my + ey - ty0) * (1.f / BH);
    const int c0 = (int)ceilf(fmaxf(lo_x, 0.f)), c1 = (int)floorf(fminf(hi_x, (float)(L::kPerRow - 1)));
    const int r0 = (int)ceilf(fmaxf(lo_y, 0.f)), r1 = (int)floorf(fminf(hi_y, (float)(L::kRows - 1)));
    if (c0 > c1 || r0 > r1) return 0u;
    const uint32_t cols = ((2u << (c1 - c0)) - 1u) << c0;
    uint32_t m = 0u;
    for (int r = r0; r <= r1; r++) m |= cols << (r * L::kPerRow);
    return m;
}

template <int kChunk>
__device__ __forceinline__ void long_fold(LongSmem<kChunk>& sm, uint32_t j, float w, bool stats)
{
    if (w > 0.f) {
        atomicMax(&sm.wmax[j], __float_as_uint(w));
        if (stats) {
            atomicAdd(&sm.ksum[j], w);
            atomicAdd(&sm.kcnt[j], 1u);
        }
    }
}

// Bands group * kGroup .. group * kGroup + kGroup - 1 of one long tile by one
// CTA; warp w renders band group * kGroup + w.
template <int BW, int BH>
__device__ __forceinline__ void render_long_tile(LongSmem<LongTile<BW, BH>::kChunk>& sm, const TileArgs& a,
                                                 int tile, int group)
{
    using L = LongTile<BW, BH>;
    constexpr int kPix = L::kPix, kSlots = L::kSlots, kPer = L::kPer, kChunk = L::kChunk;
    const int tid = threadIdx.x, lane = tid & 31, band = group * L::kGroup + (tid >> 5);
    const int W = a.W, H = a.H;
    const int gx = (W + kTileX - 1) / kTileX;
    const int bx = tile % gx, by = tile / gx;
    const float tx0 = (float)(bx * kTileX), ty0 = (float)(by * kTileY);
    const int ox = bx * kTileX + (band % L::kPerRow) * BW, oy = by * kTileY + (band / L::kPerRow) * BH;
    const int pix_lane = lane % kPix, slot = lane / kPix;
    const bool mine = lane < kPix;  // the pixel's owner lane keeps its state
    const int px = ox + pix_lane % BW, py = oy + pix_lane / BW;
    const uint2 range = a.ranges[tile];
    const uint32_t n = range.y - range.x;
    const bool stats = a.kv_sum != nullptr;
    const PairRecord* recs = a.recs + range.x;
    const float pxf = (float)px, pyf = (float)py;
    float T = 1.0f, C[3] = {0.f, 0.f, 0.f}, wmax = 0.f;
    uint32_t last = 0;
    int maxid = -1;
    bool done = !(mine && px < W && py < H);

    // A contributing record's per-chunk sums leave through global atomics; slot i
    // of chunk cbase is flushed by the thread that staged it, before it restages
    // the slot (no other thread touches the slot between the barriers around the
    // compositing).
    auto flush = [&](uint32_t cbase) {
#pragma unroll
        for (int q = 0; q < kPer; q++) {
            const int i = q * L::kThreads + tid;
            const uint32_t e = cbase + (uint32_t)i;
            if (e >= n) continue;
            const uint32_t wm = sm.wmax[i];
            if (wm && a.out_point_weight)
                atomicMax(reinterpret_cast<unsigned*>(a.out_point_weight) + __float_as_int(sm.rec[i].c.y), wm);
            if (stats && sm.kcnt[i]) {
                atomicAdd(a.kv_sum + range.x + e, sm.ksum[i]);
                atomicAdd(a.kv_cnt + range.x + e, sm.kcnt[i]);
            }
        }
    };
    PairRecord nxt[kPer];
#pragma unroll
    for (int q = 0; q < kPer; q++)
        if ((uint32_t)(q * L::kThreads + tid) < n) nxt[q] = recs[q * L::kThreads + tid];
    uint32_t last_c = 0;
    bool pending = false;
    for (uint32_t c0 = 0; c0 < n; c0 += kChunk) {
        if (pending) flush(last_c);
#pragma unroll
        for (int q = 0; q < kPer; q++) {
            const int i = q * L::kThreads + tid;
            const uint32_t e = c0 + (uint32_t)i;
            const bool have = e < n;
            if (have) sm.rec[i] = nxt[q];
            sm.mask[i] = have ? band_mask<BW, BH>(nxt[q].a, nxt[q].b, tx0, ty0) : 0u;
            sm.wmax[i] = 0u;
            if (stats) {
                sm.ksum[i] = 0.f;
                sm.kcnt[i] = 0u;
            }
            if (e + kChunk < n) nxt[q] = recs[e + kChunk];  // in flight while this chunk is composited
        }
        __syncthreads();
        for (int k = 0; k < kChunk / 32 && !__all_sync(0xffffffffu, done); k++) {
            uint32_t live = __ballot_sync(0xffffffffu, (sm.mask[k * 32 + lane] >> band) & 1u);
            const PairRecord* R = sm.rec + k * 32;
            const uint32_t k0 = c0 + (uint32_t)(k * 32);  // tile position of R[0]
            if constexpr (kSlots == 1) {
                while (live) {
                    const uint32_t j1 = (uint32_t)(__ffs(live) - 1);
                    live &= live - 1;
                    const bool two = live != 0;
                    const uint32_t j2 = two ? (uint32_t)(__ffs(live) - 1) : j1;
                    if (two) live &= live - 1;
                    const float4 ra1 = R[j1].a, rb1 = R[j1].b, ra2 = R[j2].a, rb2 = R[j2].b;
                    const float al1 = done ? 0.f : fwd_alpha(ra1, rb1, pxf, pyf);
                    const float al2 = (done || !two) ? 0.f : fwd_alpha(ra2, rb2, pxf, pyf);
                    long_fold(sm, k * 32 + j1,
                              fwd_accumulate(al1, rb1, R[j1], k0 + j1 + 1, T, C, wmax, maxid, last, done), stats);
                    long_fold(sm, k * 32 + j2,
                              fwd_accumulate(al2, rb2, R[j2], k0 + j2 + 1, T, C, wmax, maxid, last, done), stats);
                }
            } else {
                while (live) {
                    // the next kSlots live records, in order (32: none); lanes of slot s
                    // evaluate record js[s] at their pixel
                    uint32_t js[kSlots];
                    uint32_t mj = 32u;
#pragma unroll
                    for (int s = 0; s < kSlots; s++) {
                        js[s] = live ? (uint32_t)(__ffs(live) - 1) : 32u;
                        live &= live - 1;
                        if (s == slot) mj = js[s];
                    }
                    const bool pdone = __shfl_sync(0xffffffffu, done, pix_lane);
                    const float al = (mj < 32u && !pdone) ? fwd_alpha(R[mj].a, R[mj].b, pxf, pyf) : 0.f;
#pragma unroll
                    for (int s = 0; s < kSlots; s++) {
                        const float as = __shfl_sync(0xffffffffu, al, s * kPix + pix_lane);
                        const uint32_t j = js[s];
                        if (j < 32u)
                            long_fold(sm, k * 32 + j,
                                      fwd_accumulate(as, R[j].b, R[j], k0 + j + 1, T, C, wmax, maxid, last, done),
                                      stats);
                    }
                }
            }
        }
        last_c = c0;
        pending = true;
        // every pixel of this band group done: no later record can contribute (also
        // the barrier before the next chunk's staging)
        if (__syncthreads_and(done)) break;
    }
    if (pending) flush(last_c);
    if (mine && px < W && py < H) {
        const int pix = W * py + px;
        a.final_T[pix] = T;
        a.n_contrib[pix] = last;
        a.out_color[pix] = __fmaf_rn(T, a.bg[0], C[0]);
        a.out_color[H * W + pix] = __fmaf_rn(T, a.bg[1], C[1]);
        a.out_color[2 * H * W + pix] = __fmaf_rn(T, a.bg[2], C[2]);
        if (a.out_point_id) a.out_point_id[pix] = maxid;
        if (a.out_pw_pixel) a.out_pw_pixel[pix] = wmax;
    }
}

__device__ __forceinline__ void long_tile_push(uint32_t n, uint32_t id, uint32_t cap, uint32_t* __restrict__ list,
                                               uint32_t* __restrict__ ctr)
{
    const int b = 31 - __clz(n);
    const uint32_t slot = atomicAdd(ctr + 2 + b, 1u);
    list[(size_t)b * cap + slot] = id;
    atomicAdd(ctr, 1u);
}

// The long tiles of one view (ids are tiles) or of a multi-view batch (ids are
// global work items, mapped to (view, tile) by begin[]).  ctr: [0] long tiles,
// [1] tile queue, [2 + b] tiles in bin b.
__global__ void long_tiles_kernel(const uint2* __restrict__ ranges, uint32_t num_tiles, uint32_t split_min,
                                  uint32_t* __restrict__ list, uint32_t* __restrict__ ctr)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_tiles) return;
    const uint2 r = ranges[t];
    if (r.y - r.x >= split_min) long_tile_push(r.y - r.x, t, num_tiles, list, ctr);
}

__global__ void long_tiles_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin,
                                        int nviews, uint32_t total, uint32_t split_min, uint32_t* __restrict__ list,
                                        uint32_t* __restrict__ ctr)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int v = view_of(begin, nviews, i);
    const uint2 r = views[v].ranges[i - begin[v]];
    if (r.y - r.x >= split_min) long_tile_push(r.y - r.x, i, total, list, ctr);
}

// The next (long tile, band group) for this CTA (thread 0), longest bins first.
// False when the queue is empty.
template <int kGroups>
__device__ __forceinline__ bool next_long_tile(uint32_t* ctr, const uint32_t* __restrict__ list, uint32_t cap,
                                               uint32_t& id, int& group)
{
    const uint32_t item = atomicAdd(ctr + 1, 1u);
    if (item >= *(volatile uint32_t*)ctr * kGroups) return false;
    uint32_t r = item / kGroups;
    group = (int)(item % kGroups);
    for (int b = kLongBuckets - 1; b >= 0; b--) {
        const uint32_t c = *(volatile uint32_t*)(ctr + 2 + b);
        if (r < c) {
            id = list[(size_t)b * cap + r];
            return true;
        }
        r -= c;
    }
    return false;
}

template <int BW, int BH>
__global__ void __launch_bounds__(LongTile<BW, BH>::kThreads)
    render_fwd_long_kernel(TileArgs a, const uint32_t* __restrict__ list, uint32_t* ctr, uint32_t cap)
{
    extern __shared__ __align__(128) unsigned char long_dyn[];
    auto& sm = *reinterpret_cast<LongSmem<LongTile<BW, BH>::kChunk>*>(long_dyn);
    __shared__ uint32_t s_id;
    __shared__ int s_ok, s_group;
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t id = 0;
            int group = 0;
            s_ok = next_long_tile<LongTile<BW, BH>::kGroups>(ctr, list, cap, id, group);
            s_id = id;
            s_group = group;
        }
        __syncthreads();
        if (!s_ok) break;
        render_long_tile<BW, BH>(sm, a, (int)s_id, s_group);
        __syncthreads();  // s_id / s_group / s_ok are rewritten for the next item
    }
}

template <int BW, int BH>
__global__ void __launch_bounds__(LongTile<BW, BH>::kThreads)
    render_fwd_long_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin, int nviews,
                                 const uint32_t* __restrict__ list, uint32_t* ctr, uint32_t cap)
{
    extern __shared__ __align__(128) unsigned char long_dyn[];
    auto& sm = *reinterpret_cast<LongSmem<LongTile<BW, BH>::kChunk>*>(long_dyn);
    __shared__ uint32_t s_id;
    __shared__ int s_ok, s_group;
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t id = 0;
            int group = 0;
            s_ok = next_long_tile<LongTile<BW, BH>::kGroups>(ctr, list, cap, id, group);
            s_id = id;
            s_group = group;
        }
        __syncthreads();
        if (!s_ok) break;
        const uint32_t id = s_id;
        const int v = view_of(begin, nviews, id);
        render_long_tile<BW, BH>(sm, views[v], (int)(id - begin[v]), s_group);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- backward
// kConsistent: the exact-gradient backward mode (FGS_BACKWARD_CONSISTENT), a
// compile-time switch so that the reference mode pays nothing for it per pixel.
template <int PPT, int kBatch, bool kConsistent>
__device__ __forceinline__ void render_bwd_tile(BwdSmem<kBatch, bwd_slots<PPT>()>& sm, const TileArgs& a, int tile,
                                                uint32_t& gb, unsigned* err)
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

    // Per pixel: the reference's accum_rec recurrence (the colour composited behind
    // the current Gaussian, backward.cu:513-520) enters dL/dalpha only through its
    // dot product with dL/dpixel, so the pixel carries that dot product (acc_dot)
    // and the previous contributor's colour dotted the same way (last_dot): the
    // same sums, regrouped, in 2 values instead of 6.
    float T[PPT], dpix[PPT][3], acc_dot[PPT], last_dot[PPT], last_alpha[PPT];
    uint32_t last[PPT];
    // the background term of dL/dalpha, -T_final (bg . dL/dpixel) / (1 - alpha): its
    // numerator per pixel (zero for a black background, and then skipped)
    float bgT[PPT];
    const float bg0 = a.bg[0], bg1 = a.bg[1], bg2 = a.bg[2];
    uint32_t my_max = 0;
#pragma unroll
    for (int k = 0; k < PPT; k++) {
        const int py = by * kTileY + ly0 + k;
        const bool inside = px < W && py < H;
        const int pix = W * py + px;
        T[k] = inside ? a.final_T[pix] : 0.f;
        last[k] = inside ? a.n_contrib[pix] : 0;
        my_max = max(my_max, last[k]);
#pragma unroll
        for (int c = 0; c < 3; c++) dpix[k][c] = inside ? a.dL_dpix[c * H * W + pix] : 0.f;
        acc_dot[k] = 0.f;
        last_dot[k] = 0.f;
        last_alpha[k] = 0.f;
        bgT[k] = -T[k] * (bg0 * dpix[k][0] + bg1 * dpix[k][1] + bg2 * dpix[k][2]);
    }
    const float pxf = (float)px;
    const float rx0 = (float)(bx * kTileX), rx1 = rx0 + (kTileX - 1);
    const float ry0 = (float)(by * kTileY + (tid >> 5) * 2 * PPT), ry1 = ry0 + (2 * PPT - 1);
    const float ddelx_dx = 0.5 * W;
    const float ddely_dy = 0.5 * H;
    // The per-pixel loop sums w = G dL/dalpha and its products with dx, dy; the
    // factors common to all of a pair's pixels (opacity, conic, -W/2, -H/2, -1/2 of
    // backward.cu:537-551) are applied once per pair when the batch is flushed.
    // Each warp total sits on the lanes of its component.
    const int q_lane = (tid & 1) ? 15 : sum9_component((unsigned)tid);

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
                    // G and alpha in the forward's arithmetic (fwd_alpha): the same
                    // bits, so this pass skips exactly the pairs the forward skipped
                    const float dx = ra.x - pxf, dy = ra.y - (float)(by * kTileY + ly0 + k);
                    const float qf = __fmaf_rn(__fmul_rn(ra.z, dx), dx, __fmul_rn(__fmul_rn(rb.x, dy), dy));
                    const float power = __fmaf_rn(-0.5f, qf, -__fmul_rn(__fmul_rn(ra.w, dx), dy));
                    if (power > 0.0f) continue;
                    const float G = expf(power);
                    const float oG = __fmul_rn(rb.y, G);
                    const float alpha = fminf(0.99f, oG);
                    if (alpha < 1.0f / 255.0f) continue;
                    // transmittance before this Gaussian (fast reciprocal: 1 - alpha >= 0.01)
                    const float inv_1ma = __fdividef(1.f, 1.f - alpha);
                    T[k] = T[k] * inv_1ma;
                    const float dchannel_dcolor = alpha * T[k];
                    const float c2 = R[j].c.x;
                    gr[0] += dchannel_dcolor * dpix[k][0];
                    gr[1] += dchannel_dcolor * dpix[k][1];
                    gr[2] += dchannel_dcolor * dpix[k][2];
                    const float cdot = rb.z * dpix[k][0] + rb.w * dpix[k][1] + c2 * dpix[k][2];
                    acc_dot[k] += last_alpha[k] * (last_dot[k] - acc_dot[k]);
                    last_dot[k] = cdot;
                    last_alpha[k] = alpha;
                    float dL_dalpha = (cdot - acc_dot[k]) * T[k];
                    // background term; exactly zero (and skipped) for a black background
                    if (bgT[k] != 0.f) dL_dalpha += bgT[k] * inv_1ma;
                    if (kConsistent && oG > 0.99f) dL_dalpha = 0.f;
                    // w = G dL/dalpha = dL/dopacity; w dx and w dy give dL/dmean2D,
                    // w dx dx, w dx dy and w dy dy dL/dconic (times the pair's factors)
                    const float w = G * dL_dalpha;
                    const float u = w * dx, v = w * dy;
                    gr[3] += u;
                    gr[4] += v;
                    gr[5] += u * dx;
                    gr[6] += u * dy;
                    gr[7] += v * dy;
                    gr[8] += w;
                    any = true;
                }
                if (__any_sync(0xffffffffu, any)) {
                    const float tot = warp_transpose_sum9(gr);
                    if (q_lane < NG) atomicAdd(&sm.acc[(tid >> 5) >> 1][q_lane][j], tot);
                }
            }
        }
        __syncthreads();
        // this batch's per-pair gradients, at each pair's emission index: the slot
        // sums times the pair's own factors
        for (uint32_t e = tid; e < cnt; e += NT) {
            float* dst = a.pgrad + (size_t)__float_as_uint(R[e].c.w) * NG;
            float sum[NG];
#pragma unroll
            for (int q = 0; q < NG; q++) {
                float v = 0.f;
#pragma unroll
                for (int sl = 0; sl < kSlots; sl++) {
                    v += sm.acc[sl][q][e];
                    sm.acc[sl][q][e] = 0.f;
                }
                sum[q] = v;
            }
            const float4 ea = R[e].a, eb = R[e].b;  // conic (ea.z, ea.w, eb.x), opacity eb.y
            const float o = eb.y;
            dst[0] = sum[0];
            dst[1] = sum[1];
            dst[2] = sum[2];
            dst[3] = -ddelx_dx * (o * (ea.z * sum[3] + ea.w * sum[4]));
            dst[4] = -ddely_dy * (o * (eb.x * sum[4] + ea.w * sum[3]));
            dst[5] = -0.5f * (o * sum[5]);
            dst[6] = -0.5f * (o * sum[6]);
            dst[7] = -0.5f * (o * sum[7]);
            dst[8] = sum[8];
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

// Resident CTAs per SM the multi-view backward is compiled for: 32 warps at 2 pixels
// per thread (64 registers, a few spilled bytes) and 24 at 4 (80 registers and a few
// spilled bytes instead of the 110 the compiler takes when left alone; with 64-record
// batches the shared memory then lets all 12 CTAs in).  Measured: 4 pixels per thread
// at 12 CTAs beats 10 (no spills) and 14 (more spills); 2 at 8 beats 6.  The
// single-view kernel keeps the compiler's allocation.
template <int PPT>
constexpr int bwd_multi_min_ctas() { return PPT == 2 ? 8 : (PPT == 4 ? 12 : 1); }

template <int PPT, int kBatch, bool kConsistent>
__global__ void __launch_bounds__(256 / PPT) render_bwd_kernel(TileArgs a, unsigned* err)
{
    extern __shared__ __align__(128) unsigned char bwd_dyn[];
    BwdSmemT<PPT, kBatch>& sm = *reinterpret_cast<BwdSmemT<PPT, kBatch>*>(bwd_dyn);
    bwd_smem_init(sm, 256 / PPT);
    uint32_t gb = 0;
    render_bwd_tile<PPT, kBatch, kConsistent>(sm, a, blockIdx.x, gb, err);
}

template <int PPT, int kBatch, bool kConsistent>
__global__ void __launch_bounds__(256 / PPT, bwd_multi_min_ctas<PPT>())
    render_bwd_multi_kernel(const TileArgs* __restrict__ views, const uint32_t* __restrict__ begin, int nviews,
                            uint32_t total, uint32_t* queue, unsigned* err)
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
        const TileArgs& a = views[v];  // fields read where used, not held in registers
        render_bwd_tile<PPT, kBatch, kConsistent>(sm, a, (int)(item - begin[v]), gb, err);
        __syncthreads();
    }
}

}  // namespace

namespace {
RenderConfig g_cfg{2, 256, 2, 256, 0, 0};

// Dynamic shared memory of a forward launch: the whole FwdSmem with statistics,
// up to its statistics sums without.
template <int kBatch>
size_t fwd_smem_bytes(bool stats)
{
    return stats ? sizeof(FwdSmem<kBatch>) : offsetof(FwdSmem<kBatch>, ksum);
}

// Dynamic shared memory of a long-tile kernel (opted in once per process and device
// ordinal; Tag tells the kernels apart: single-view 0, multi-view 1).
template <int BW, int BH, int Tag, typename Kern>
size_t long_smem_bytes(Kern k)
{
    static bool done[64] = {};
    const size_t bytes = sizeof(LongSmem<LongTile<BW, BH>::kChunk>);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !done[dev]) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (dev >= 0 && dev < 64) done[dev] = true;
    }
    return bytes;
}

// Band shapes (fgs_set_render_split): 0 = 16x2, 1 = 8x4, 2 = 4x4, 3 = 4x2 pixels per warp.
template <int BW, int BH>
void long_launch(const TileArgs& a, const uint32_t* list, uint32_t* ctr, uint32_t cap, cudaStream_t s)
{
    constexpr int kThreads = LongTile<BW, BH>::kThreads;
    const size_t smem = long_smem_bytes<BW, BH, 0>(render_fwd_long_kernel<BW, BH>);
    render_fwd_long_kernel<BW, BH><<<resident_ctas(render_fwd_long_kernel<BW, BH>, kThreads), kThreads, smem, s>>>(
        a, list, ctr, cap);
}
void launch_long_kernel(int shape, const TileArgs& a, const uint32_t* list, uint32_t* ctr, uint32_t cap,
                        cudaStream_t s)
{
    if (shape == 1) long_launch<8, 4>(a, list, ctr, cap, s);
    else if (shape == 2) long_launch<4, 4>(a, list, ctr, cap, s);
    else if (shape == 3) long_launch<4, 2>(a, list, ctr, cap, s);
    else long_launch<16, 2>(a, list, ctr, cap, s);
}
template <int BW, int BH>
void long_multi_launch(const TileArgs* views, const uint32_t* begin, int nviews, const uint32_t* list, uint32_t* ctr,
                       uint32_t cap, cudaStream_t s)
{
    constexpr int kThreads = LongTile<BW, BH>::kThreads;
    const size_t smem = long_smem_bytes<BW, BH, 1>(render_fwd_long_multi_kernel<BW, BH>);
    render_fwd_long_multi_kernel<BW, BH>
        <<<resident_ctas(render_fwd_long_multi_kernel<BW, BH>, kThreads), kThreads, smem, s>>>(views, begin, nviews,
                                                                                             list, ctr, cap);
}
void launch_long_multi_kernel(int shape, const TileArgs* views, const uint32_t* begin, int nviews,
                              const uint32_t* list, uint32_t* ctr, uint32_t cap, cudaStream_t s)
{
    if (shape == 1) long_multi_launch<8, 4>(views, begin, nviews, list, ctr, cap, s);
    else if (shape == 2) long_multi_launch<4, 4>(views, begin, nviews, list, ctr, cap, s);
    else if (shape == 3) long_multi_launch<4, 2>(views, begin, nviews, list, ctr, cap, s);
    else long_multi_launch<16, 2>(views, begin, nviews, list, ctr, cap, s);
}

template <int PPT, int B>
void fwd_launch(int grid, const ImageState& im, const BinState& b, long long K, int W, int H, const float* bg,
                float* out_color, int* point_id, float* pw_pixel, float* point_weight, bool stats, int split,
                int band_shape, unsigned* err, cudaStream_t s)
{
    TileArgs a{};
    a.ranges = im.ranges; a.recs = b.rec; a.W = W; a.H = H; a.bg = bg;
    a.out_color = out_color; a.final_T = im.final_T; a.n_contrib = im.n_contrib; a.out_point_id = point_id;
    a.out_pw_pixel = pw_pixel; a.out_point_weight = point_weight;
    a.kv_sum = stats ? b.kv_sum : nullptr; a.kv_cnt = stats ? b.kv_cnt : nullptr;
    if (split > 0) {
        // long tiles first, in bands; the tile kernel then skips them
        cudaMemsetAsync(im.long_ctr, 0, (2 + kLongBuckets) * sizeof(uint32_t), s);
        if (stats && K > 0) {
            cudaMemsetAsync(b.kv_sum, 0, sizeof(float) * (size_t)K, s);
            cudaMemsetAsync(b.kv_cnt, 0, sizeof(uint32_t) * (size_t)K, s);
        }
        long_tiles_kernel<<<(grid + 255) / 256, 256, 0, s>>>(im.ranges, (uint32_t)grid, (uint32_t)split, im.long_list,
                                                             im.long_ctr);
        launch_long_kernel(band_shape, a, im.long_list, im.long_ctr, (uint32_t)grid, s);
        note_launches(2);
    }
    render_fwd_kernel<PPT, B><<<grid, 256 / PPT, fwd_smem_bytes<B>(stats), s>>>(a, (uint32_t)(split > 0 ? split : 0),
                                                                                err);
}

// Dynamic shared memory of a backward kernel instantiation (opted in once per process
// and device ordinal; Tag tells the kernels apart: single-view 0, multi-view 1, +2 in the
// consistent mode).
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
    if (consistent) {
        const size_t smem = bwd_smem_bytes<PPT, B, 2>(render_bwd_kernel<PPT, B, true>);
        render_bwd_kernel<PPT, B, true><<<grid, 256 / PPT, smem, s>>>(a, err);
    } else {
        const size_t smem = bwd_smem_bytes<PPT, B, 0>(render_bwd_kernel<PPT, B, false>);
        render_bwd_kernel<PPT, B, false><<<grid, 256 / PPT, smem, s>>>(a, err);
    }
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
    return ok_p(c.fwd_ppt) && ok_p(c.bwd_ppt) && ok_b(c.fwd_batch) && ok_b(c.bwd_batch) && c.fwd_split >= 0 &&
           c.fwd_band >= 0 && c.fwd_band <= 3;
}
void set_render_config(const RenderConfig& c) { g_cfg = c; }
RenderConfig get_render_config() { return g_cfg; }

void launch_render_fwd(int W, int H, const ImageState& im, const BinState& b, long long K, const float* bg,
                       float* out_color, int* point_id, float* pw_pixel, float* point_weight, bool stats,
                       unsigned* err, cudaStream_t s)
{
    const int gx = (W + kTileX - 1) / kTileX, gy = (H + kTileY - 1) / kTileY;
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(fwd_launch, c.fwd_ppt, c.fwd_batch, gx * gy, im, b, K, W, H, bg, out_color, point_id,
                        pw_pixel, point_weight, stats, c.fwd_split, c.fwd_band, err, s);
    note_launches(1);
}

namespace {
template <int PPT, int B>
void fwd_multi_launch(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total, uint32_t* queue,
                      uint32_t* long_list, uint32_t* long_ctr, int split, int band_shape, unsigned* err,
                      cudaStream_t s)
{
    if (split > 0) {
        cudaMemsetAsync(long_ctr, 0, (2 + kLongBuckets) * sizeof(uint32_t), s);
        long_tiles_multi_kernel<<<(total + 255) / 256, 256, 0, s>>>(views, begin, nviews, total, (uint32_t)split,
                                                                    long_list, long_ctr);
        launch_long_multi_kernel(band_shape, views, begin, nviews, long_list, long_ctr, total, s);
        note_launches(2);
    }
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = fwd_smem_bytes<B>(false);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_fwd_multi_kernel<PPT, B>, 256 / PPT, smem);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    render_fwd_multi_kernel<PPT, B><<<grid, 256 / PPT, smem, s>>>(views, begin, nviews, total, queue,
                                                               (uint32_t)(split > 0 ? split : 0), err);
}

template <int PPT, int B, bool kConsistent>
void bwd_multi_launch_mode(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total, uint32_t* queue,
                           unsigned* err, cudaStream_t s)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = bwd_smem_bytes<PPT, B, kConsistent ? 3 : 1>(render_bwd_multi_kernel<PPT, B, kConsistent>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_bwd_multi_kernel<PPT, B, kConsistent>, 256 / PPT,
                                                  smem);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    render_bwd_multi_kernel<PPT, B, kConsistent><<<grid, 256 / PPT, smem, s>>>(views, begin, nviews, total, queue,
                                                                               err);
}

template <int PPT, int B>
void bwd_multi_launch(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total, uint32_t* queue,
                      int consistent, unsigned* err, cudaStream_t s)
{
    if (consistent) bwd_multi_launch_mode<PPT, B, true>(views, begin, nviews, total, queue, err, s);
    else bwd_multi_launch_mode<PPT, B, false>(views, begin, nviews, total, queue, err, s);
}
}  // namespace

void launch_render_fwd_multi(const TileArgs* views, const uint32_t* begin, int nviews, uint32_t total_tiles,
                             uint32_t* queue, uint32_t* long_list, uint32_t* long_ctr, unsigned* err, cudaStream_t s)
{
    cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    const RenderConfig c = g_cfg;
    FGS_RENDER_DISPATCH(fwd_multi_launch, c.fwd_ppt, c.fwd_batch, views, begin, nviews, total_tiles, queue, long_list,
                        long_ctr, c.fwd_split, c.fwd_band, err, s);
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
