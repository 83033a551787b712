// Per-Gaussian forward preprocess and the radius / visibility kernels.
//
// preprocess: antialias/cuda_rasterizer/forward.cu:266-401 (EWA projection,
// 2D dilation, OGFS opacity-aware radius, tile rectangle, SH degree<=3
// colour), plus the optional 3D filter, in two passes: a cheap pass over all P
// Gaussians (near plane, and a conservative bound on the tile rectangle that
// needs no projection of the covariance) appends the few that may touch a
// tile to a candidate list, and the exact path then runs over the candidates
// on dense warps.  (In one pass, the ~6% visible Gaussians of a typical view
// spread over nearly every warp and every warp pays for the exact path.)
//
// Radii and tiles-touched are written for every Gaussian.  Only the V
// visible ones (tiles > 0) get the 48-byte render record and SH clamp bits.
// They are then compacted in index order -- ids into sort_ids_b, depth bits
// into depth_key -- by reduce-then-scan over chunks of 256 ids: the exact pass
// adds to its chunk's visible and pair counts, one CTA scans the chunk counts
// (and writes K and V to the device), and a scatter pass places the ids.  The
// depth sort then runs over V keys instead of P with the same result: equal
// depths keep index order.
#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr int kThreads = 256;

// Per-Gaussian inputs: from the packed structure-of-arrays copy when there is one
// (one float4 per plane), else from the reference's AoS tensors.
__device__ __forceinline__ float3 in_mean(const PreParams& p, int idx)
{
    if (p.packed) {
        const float4 v = __ldg(p.packed + idx);
        return {v.x, v.y, v.z};
    }
    return {__ldg(p.means + 3 * (size_t)idx), __ldg(p.means + 3 * (size_t)idx + 1),
            __ldg(p.means + 3 * (size_t)idx + 2)};
}
__device__ __forceinline__ float in_opacity(const PreParams& p, int idx)
{
    return p.packed ? __ldg(p.packed + idx).w : __ldg(p.opac + idx);
}
__device__ __forceinline__ float3 in_scale(const PreParams& p, int idx)
{
    if (p.packed) {
        const float4 v = __ldg(p.packed + (size_t)p.P + idx);
        return {v.x, v.y, v.z};
    }
    return {__ldg(p.scales + 3 * (size_t)idx), __ldg(p.scales + 3 * (size_t)idx + 1),
            __ldg(p.scales + 3 * (size_t)idx + 2)};
}
__device__ __forceinline__ float4 in_rot(const PreParams& p, int idx)
{
    if (p.packed) return __ldg(p.packed + 2 * (size_t)p.P + idx);
    if (p.aligned) return __ldg(reinterpret_cast<const float4*>(p.rots) + idx);
    return make_float4(__ldg(p.rots + 4 * (size_t)idx), __ldg(p.rots + 4 * (size_t)idx + 1),
                       __ldg(p.rots + 4 * (size_t)idx + 2), __ldg(p.rots + 4 * (size_t)idx + 3));
}

__global__ void pack_gaussians_kernel(int P, const float* __restrict__ means, const float* __restrict__ opac,
                                      const float* __restrict__ scales, const float* __restrict__ rots,
                                      float4* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        out[i] = make_float4(means[3 * (size_t)i], means[3 * (size_t)i + 1], means[3 * (size_t)i + 2], opac[i]);
        if (scales && rots) {
            out[(size_t)P + i] =
                make_float4(scales[3 * (size_t)i], scales[3 * (size_t)i + 1], scales[3 * (size_t)i + 2], 0.f);
            out[2 * (size_t)P + i] = make_float4(rots[4 * (size_t)i], rots[4 * (size_t)i + 1],
                                                 rots[4 * (size_t)i + 2], rots[4 * (size_t)i + 3]);
        }
    }
}

// trace(cov3D) for cov3D = M^T M, M = S R (forward.cu:151-185): the sum of the
// squared entries of M, row r of R scaled by s_r.
__device__ __forceinline__ float cov3d_trace(float sx, float sy, float sz, float mod, float4 q)
{
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    const float r0 = (1.f - 2.f * (y * y + z * z)) * (1.f - 2.f * (y * y + z * z)) +
                     4.f * ((x * y + r * z) * (x * y + r * z) + (x * z - r * y) * (x * z - r * y));
    const float r1 = (1.f - 2.f * (x * x + z * z)) * (1.f - 2.f * (x * x + z * z)) +
                     4.f * ((x * y - r * z) * (x * y - r * z) + (y * z + r * x) * (y * z + r * x));
    const float r2 = (1.f - 2.f * (x * x + y * y)) * (1.f - 2.f * (x * x + y * y)) +
                     4.f * ((x * z + r * y) * (x * z + r * y) + (y * z - r * x) * (y * z - r * x));
    const float a = mod * sx, b = mod * sy, c = mod * sz;
    return a * a * r0 + b * b * r1 + c * c * r2;
}

// Conservative tile test before the projection (skips only Gaussians whose
// exact path would touch no tile, so every output is unchanged).  With
// cov3D = M^T M positive semi-definite, lambda_max(cov3D) <= trace(cov3D), and
// the 2D covariance T^T cov3D T (T = W J, forward.cu:102-146, with the same
// clamped t.x / t.y) has trace <= trace(cov3D) (|T_0|^2 + |T_1|^2); dilation
// adds at most 0.3 per diagonal entry.  The OGFS radius is at most
// max(1, ratio_min) * 3 sqrt(lambda_max) + 1 pixels.  The 1% + 1e-4 and +1 px
// margins absorb the float rounding of the exact path.
__device__ __forceinline__ bool may_touch_tiles(const PreParams& p, float3 t, float tr3, float px, float py)
{
    const float* v = p.view;
    const float limx = 1.3f * p.tanx, limy = 1.3f * p.tany;
    const float tx = fminf(limx, fmaxf(-limx, t.x / t.z)) * t.z;
    const float ty = fminf(limy, fmaxf(-limy, t.y / t.z)) * t.z;
    const float j00 = p.fx / t.z, j20 = -(p.fx * tx) / (t.z * t.z);
    const float j11 = p.fy / t.z, j21 = -(p.fy * ty) / (t.z * t.z);
    const float a0 = j00 * v[0] + j20 * v[2], a1 = j00 * v[4] + j20 * v[6], a2 = j00 * v[8] + j20 * v[10];
    const float b0 = j11 * v[1] + j21 * v[2], b1 = j11 * v[5] + j21 * v[6], b2 = j11 * v[9] + j21 * v[10];
    const float lam = tr3 * (a0 * a0 + a1 * a1 + a2 * a2 + b0 * b0 + b1 * b1 + b2 * b2) + (p.use_filter ? 0.6f : 0.f);
    const float r = fmaxf(1.f, p.ratio_min) * 3.f * sqrtf(1.01f * lam + 1e-4f) + 2.f;
    if (!(r < 1e7f) || !(fabsf(px) < 1e9f) || !(fabsf(py) < 1e9f)) return true;  // no safe bound: exact path
    const int gx = (p.W + kTileX - 1) / kTileX, gy = (p.H + kTileY - 1) / kTileY;
    int x0, y0, x1, y1;
    tile_rect(px, py, (int)ceilf(r), gx, gy, kTileX, kTileY, x0, y0, x1, y1);
    return (x1 - x0) * (y1 - y0) != 0;
}

// Pass 1, every Gaussian: near plane and the conservative tile bound.  The
// Gaussians that fail get radius 0 / no tiles here; the rest (typically a
// small fraction of P) are appended to a candidate list, so that pass 2 --
// projection, radius, colour -- runs on dense warps instead of on the few
// live lanes of every warp.
__global__ void __launch_bounds__(kThreads) preprocess_cull_kernel(PreParams p, GeomState g,
                                                                   int* __restrict__ radii_out)
{
    // Persistent CTAs collect their candidates in shared memory and reserve room
    // in the global list once per flush: one atomic per CTA-flush instead of one
    // per warp (same-address atomics from every warp serialise at L2).
    constexpr int kList = 8 * kThreads;
    __shared__ uint32_t s_list[kList];
    __shared__ uint32_t s_wc[kThreads / 32];
    __shared__ uint32_t s_n, s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int stride = gridDim.x * kThreads;
    for (int idx0 = blockIdx.x * kThreads; idx0 < p.P; idx0 += stride) {
        const int idx = idx0 + threadIdx.x;
        bool cand = false;
        if (idx < p.P) {
            const float3 p_orig = in_mean(p, idx);
            const float3 p_view = xform_point4x3(p_orig, p.view);
            if (p_view.z <= 0.2f) {  // auxiliary.h:139-164
                if (p.prefiltered) set_error(g.err, FGS_ERR_PREFILTERED);
            } else if (p.cov3D) {
                cand = true;  // no bound for an arbitrary precomputed covariance
            } else {
                const float4 p_hom = xform_point4x4(p_orig, p.proj);
                const float p_w = 1.0f / (p_hom.w + 0.0000001f);
                const float px = ndc_to_pix(p_hom.x * p_w, p.W), py = ndc_to_pix(p_hom.y * p_w, p.H);
                const float4 q = in_rot(p, idx);
                const float3 sc = in_scale(p, idx);
                float tr = cov3d_trace(sc.x, sc.y, sc.z, p.scale_mod, q);
                if (p.filter3d > 0.f) {
                    const float sf = p.filter3d * p_view.z / p.fx;
                    tr += 3.f * sf * sf;
                }
                cand = may_touch_tiles(p, p_view, tr, px, py);
            }
            if (!cand) {
                g.tiles[idx] = 0;
                g.radii[idx] = 0;
                if (radii_out) radii_out[idx] = 0;
            }
        }
        // append to the CTA's list (the order is irrelevant: the visible set is
        // compacted in index order afterwards)
        const unsigned cb = __ballot_sync(0xffffffffu, cand);
        if (lane == 0) s_wc[warp] = __popc(cb);
        __syncthreads();
        // s_n is read once, before the barrier: thread 0 rewrites it after the
        // barrier, and every thread must take the same flush decision from n.
        const uint32_t n0 = s_n;
        uint32_t pos = n0 + __popc(cb & ((1u << lane) - 1u)), tot = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; w++) {
            if (w < warp) pos += s_wc[w];
            tot += s_wc[w];
        }
        if (cand) s_list[pos] = (uint32_t)idx;
        const uint32_t n = n0 + tot;
        __syncthreads();
        const bool last = idx0 + stride >= p.P;
        if (n > kList - kThreads || last) {
            if (threadIdx.x == 0) s_base = n ? atomicAdd(g.counters + 12, n) : 0u;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < n; k += kThreads) {
                if (s_base + k < (uint32_t)p.P) g.cand_ids[s_base + k] = s_list[k];
                else set_error(g.err, FGS_ERR_OVERFLOW);  // a list longer than P: never write past it
            }
            __syncthreads();
            if (threadIdx.x == 0) s_n = 0;
        } else if (threadIdx.x == 0) {
            s_n = n;
        }
        __syncthreads();
    }
}

// Pass 2, the candidates: the exact path (forward.cu:266-401), one Gaussian per
// thread.  Visible Gaussians add to the per-chunk (256 consecutive ids) visible
// and pair counts that the ordered compaction scans.
__global__ void __launch_bounds__(kThreads) preprocess_full_kernel(PreParams p, GeomState g,
                                                                   int* __restrict__ radii_out)
{
    __shared__ float s_log_lambda_G;
    if (threadIdx.x == 0) {
        // forward.cu:345-355: the opacity-independent part of the OGFS radius, once per CTA
        const float epsilon_pix = 1.0f / 255.0f;
        const float eps_base = fmaxf(0.0f, 1.0f - epsilon_pix);
        const float lambda_G_raw = 1.0f - powf(eps_base, static_cast<float>(kOgfsBlockArea));
        float lambda_G = epsilon_pix + p.eps_scale * (lambda_G_raw - epsilon_pix);
        lambda_G = fminf(fmaxf(lambda_G, epsilon_pix), p.eps_max);
        s_log_lambda_G = logf(lambda_G);
    }
    __syncthreads();
    const uint32_t ncand = min(*(volatile uint32_t*)(g.counters + 12), (uint32_t)p.P);
    const bool vec = p.aligned != 0;
    for (uint32_t k = blockIdx.x * kThreads + threadIdx.x; k < ncand; k += gridDim.x * kThreads) {
        const int idx = (int)g.cand_ids[k];
        uint32_t tiles = 0;
        int radius_px = 0;
        uint8_t clamp_bits = 0;
        PairRecord rec;
        const float3 p_orig = in_mean(p, idx);
        const float4 p_hom = xform_point4x4(p_orig, p.proj);
        const float p_w = 1.0f / (p_hom.w + 0.0000001f);
        const float3 p_proj = {p_hom.x * p_w, p_hom.y * p_w, p_hom.z * p_w};
        const float3 p_view = xform_point4x3(p_orig, p.view);
        const float px = ndc_to_pix(p_proj.x, p.W), py = ndc_to_pix(p_proj.y, p.H);
        float cov3D[6];
        if (p.cov3D) {
#pragma unroll
            for (int c = 0; c < 6; c++) cov3D[c] = __ldg(p.cov3D + (size_t)idx * 6 + c);
        } else {
            const float4 q = in_rot(p, idx);
            const float3 sc = in_scale(p, idx);
            cov3d_ref(sc.x, sc.y, sc.z, p.scale_mod, q, cov3D);
        }
        if (p.filter3d > 0.f) {
            // 3D filter: isotropic variance of a sigma = s * z / focal blur, added as its own
            // rounded terms (what feeding the filtered covariance to the reference gives)
            const float sf = __fdiv_rn(__fmul_rn(p.filter3d, p_view.z), p.fx);
            const float v = __fmul_rn(sf, sf);
            cov3D[0] = __fadd_rn(cov3D[0], v); cov3D[3] = __fadd_rn(cov3D[3], v); cov3D[5] = __fadd_rn(cov3D[5], v);
        }
        float3 cov = ewa_cov2d_ref(p_orig, p.fx, p.fy, p.tanx, p.tany, cov3D, p.view);
        if (p.use_filter) {
            cov.x = dilate_max(cov.x);
            cov.z = dilate_max(cov.z);
        }
        // forward.cu:328-330, the first product fused as in the reference build
        const float det = __fmaf_rn(cov.x, cov.z, -__fmul_rn(cov.y, cov.y));
        if (det != 0.0f) {
            const float det_inv = __fdiv_rn(1.f, det);
            const float3 conic = {__fmul_rn(cov.z, det_inv), __fmul_rn(-cov.y, det_inv), __fmul_rn(cov.x, det_inv)};
            // forward.cu:345-369: OGFS radius
            const float opacity = fmaxf(in_opacity(p, idx), 1e-6f);
            const float log_opacity = logf(opacity);
            const float radius_energy = log_opacity - s_log_lambda_G;
            const float energy_clamped = fmaxf(radius_energy, p.energy_floor);
            const float mid = 0.5f * (cov.x + cov.z);
            const float disc = fmaxf(0.0f, mid * mid - det);
            const float sqrt_disc = sqrtf(disc);
            const float lambda1 = mid + sqrt_disc;
            const float lambda2 = mid - sqrt_disc;
            const float max_lambda = fmaxf(fmaxf(lambda1, lambda2), 1e-6f);
            const float radius_base = 3.0f * sqrtf(max_lambda);
            float radius_major = sqrtf(2.0f * energy_clamped * max_lambda);
            radius_major = fminf(radius_major, radius_base);
            radius_major = fmaxf(radius_major, p.ratio_min * radius_base);
            const float radius_f = radius_major + 1.0f;
            const int rpx = max(1, static_cast<int>(ceilf(radius_f)));
            const int gx = (p.W + kTileX - 1) / kTileX, gy = (p.H + kTileY - 1) / kTileY;
            int x0, y0, x1, y1;
            tile_rect(px, py, rpx, gx, gy, kTileX, kTileY, x0, y0, x1, y1);
            const int extent = (x1 - x0) * (y1 - y0);
            if (extent != 0) {
                float3 rgb;
                if (p.colors) {
                    rgb = {__ldg(p.colors + 3 * (size_t)idx), __ldg(p.colors + 3 * (size_t)idx + 1),
                           __ldg(p.colors + 3 * (size_t)idx + 2)};
                } else {
                    // SH row: 12 float4 loads when the row is 16-byte aligned.
                    float sh[48];
                    const int nf = p.M * 3;
                    const float* row = p.shs + (size_t)idx * nf;
                    const int ncoef = (p.D + 1) * (p.D + 1);
                    const int need = min(nf, ncoef * 3);
                    if (vec && (nf & 3) == 0) {
                        const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
                        for (int v = 0; v < 12; v++)
                            if (4 * v < need) {
                                const float4 q = __ldg(r4 + v);
                                sh[4 * v] = q.x; sh[4 * v + 1] = q.y; sh[4 * v + 2] = q.z; sh[4 * v + 3] = q.w;
                            }
                    } else {
#pragma unroll
                        for (int f = 0; f < 48; f++)
                            if (f < need) sh[f] = __ldg(row + f);
                    }
                    const float3 cam = {__ldg(p.campos), __ldg(p.campos + 1), __ldg(p.campos + 2)};
                    rgb = sh_to_rgb(p.D, sh, p_orig, cam, clamp_bits);
                }
                radius_px = rpx;
                tiles = (uint32_t)extent;
                rec.a = make_float4(px, py, conic.x, conic.y);
                rec.b = make_float4(conic.z, opacity, rgb.x, rgb.y);
                rec.c = make_float4(rgb.z, __int_as_float(idx), p_view.z, 0.f);
            }
        }
        if (tiles) {
            g.grec[idx] = rec;
            g.clamped[idx] = clamp_bits;
            const uint32_t nch = (uint32_t)((p.P + kThreads - 1) / kThreads);
            atomicAdd(g.chunk_counts + idx / kThreads, 1u);
            atomicAdd(g.chunk_counts + nch + idx / kThreads, tiles);
        }
        g.tiles[idx] = tiles;
        g.radii[idx] = radius_px;
        if (radii_out) radii_out[idx] = radius_px;
    }
}

// Exclusive scan of the per-chunk visible counts (in place) and the totals
// K = sum of pair counts, V = sum of visible counts.  One CTA of 1024 threads,
// each owning a contiguous run of chunks.
__global__ void __launch_bounds__(1024) chunk_scan_kernel(uint32_t* __restrict__ counts, uint32_t nch,
                                                         unsigned long long* __restrict__ total)
{
    // Up to kReg chunks per thread are held in registers, so all loads are in
    // flight at once (P <= 1024 * kReg * 256 = 4M); larger P loops.
    constexpr int kReg = 16;
    __shared__ unsigned long long s_v[32], s_k[32];
    const uint32_t per = (nch + 1023) / 1024;
    const uint32_t b = min(nch, threadIdx.x * per), e = min(nch, b + per);
    unsigned long long sv = 0, sk = 0;
    uint32_t v[kReg];
    if (per <= (uint32_t)kReg) {
#pragma unroll
        for (int i = 0; i < kReg; i++) {
            v[i] = b + i < e ? counts[b + i] : 0u;
            sk += b + i < e ? counts[nch + b + i] : 0u;
        }
#pragma unroll
        for (int i = 0; i < kReg; i++) sv += v[i];
    } else {
        for (uint32_t i = b; i < e; i++) {
            sv += counts[i];
            sk += counts[nch + i];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = sv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sk += __shfl_xor_sync(0xffffffffu, sk, o);
    if (lane == 31) s_v[warp] = x;
    if (lane == 0) s_k[warp] = sk;
    __syncthreads();
    unsigned long long wpre = 0, vtot = 0, ktot = 0;
    for (int w = 0; w < 32; w++) {
        if (w < warp) wpre += s_v[w];
        vtot += s_v[w];
        ktot += s_k[w];
    }
    unsigned long long excl = wpre + x - sv;
    if (per <= (uint32_t)kReg) {
#pragma unroll
        for (int i = 0; i < kReg; i++)
            if (b + i < e) {
                counts[b + i] = (uint32_t)excl;
                excl += v[i];
            }
    } else {
        for (uint32_t i = b; i < e; i++) {
            const uint32_t c = counts[i];
            counts[i] = (uint32_t)excl;
            excl += c;
        }
    }
    if (threadIdx.x == 0) {
        total[0] = ktot;
        total[1] = vtot;
    }
}

// Ordered scatter of the visible ids and their depth bits (the view depth kept
// in the render record).
__global__ void __launch_bounds__(kThreads) compact_visible_kernel(int P, const uint32_t* __restrict__ tiles,
                                                                   const PairRecord* __restrict__ grec,
                                                                   const uint32_t* __restrict__ chunk_prefix,
                                                                   uint32_t* __restrict__ ids,
                                                                   uint32_t* __restrict__ keys)
{
    __shared__ uint32_t s_wv[kThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int idx = blockIdx.x * kThreads + t;
    const bool vis = idx < P && __ldg(tiles + idx) != 0;
    const unsigned vb = __ballot_sync(0xffffffffu, vis);
    if (lane == 0) s_wv[warp] = __popc(vb);
    __syncthreads();
    uint32_t pos = __ldg(chunk_prefix + blockIdx.x) + __popc(vb & ((1u << lane) - 1u));
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++)
        if (w < warp) pos += s_wv[w];
    if (vis) {
        ids[pos] = (uint32_t)idx;
        keys[pos] = __float_as_uint(grec[idx].c.z);
    }
}

// forward.cu:187-263 (variant 0) and compute_radius_kernel_v2.cu:180-229 (variant 1)
__global__ void compute_radius_kernel(int variant, int P, const float* __restrict__ means,
                                      const float* __restrict__ scales, const float* __restrict__ rots,
                                      const float* __restrict__ view, const float* __restrict__ proj, float fx,
                                      float fy, float tanx, float tany, float* __restrict__ radius)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    radius[idx] = 0;
    const float3 p_orig = {means[3 * idx], means[3 * idx + 1], means[3 * idx + 2]};
    const float4 p_hom = xform_point4x4(p_orig, proj);
    const float p_w = 1.0f / (p_hom.w + 0.0000001f);
    const float3 p_proj = {p_hom.x * p_w, p_hom.y * p_w, p_hom.z * p_w};
    if (variant == 0) {
        const float3 p_view = xform_point4x3(p_orig, view);
        if (p_view.z <= 0.2f) return;
    }
    if (p_proj.x < -1.3 || p_proj.x > 1.3 || p_proj.y < -1.3 || p_proj.y > 1.3) return;
    float cov3D[6];
    const float4 q = {rots[4 * idx], rots[4 * idx + 1], rots[4 * idx + 2], rots[4 * idx + 3]};
    cov3d_from_scale_rot(scales[3 * idx], scales[3 * idx + 1], scales[3 * idx + 2], 1.f, q, cov3D);
    float3 cov = ewa_cov2d(p_orig, fx, fy, tanx, tany, cov3D, view);
    if (variant == 1) {
        cov.x = dilate_max(cov.x);
        cov.z = dilate_max(cov.z);
    }
    const float det = (cov.x * cov.z - cov.y * cov.y);
    if (det == 0.0f) return;
    const float mid = 0.5f * (cov.x + cov.z);
    const float lambda1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float lambda2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
    radius[idx] = 3.f * sqrtf(fmaxf(lambda1, lambda2));
}

// rasterizer_impl.cu:97-109
__global__ void mark_visible_kernel(int P, const float* __restrict__ means, const float* __restrict__ view,
                                    uint8_t* __restrict__ present)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    const float3 p = {means[3 * idx], means[3 * idx + 1], means[3 * idx + 2]};
    present[idx] = xform_point4x3(p, view).z > 0.2f;
}

// compute_radius_kernel_v2.cu:109-169
__device__ __forceinline__ bool vis_radius_point(int idx, const float* __restrict__ means,
                                                 const float* __restrict__ lscales, const float* __restrict__ rots,
                                                 const float* __restrict__ proj, const float* __restrict__ view,
                                                 float fx, float fy, float tanx, float tany, float padding,
                                                 float& depth_out, float& radius_out)
{
    const float3 p_orig = {means[3 * idx], means[3 * idx + 1], means[3 * idx + 2]};
    const float4 p_hom = xform_point4x4(p_orig, proj);
    const float p_w = 1.0f / (p_hom.w + 0.0000001f);
    const float3 p_proj = {p_hom.x * p_w, p_hom.y * p_w, p_hom.z * p_w};
    depth_out = p_proj.z;
    const bool visible = (p_proj.z > 0.0f) && (p_proj.z < 1.0f) && (p_proj.x > -1.0f - padding) &&
                         (p_proj.x < 1.0f + padding) && (p_proj.y > -1.0f - padding) && (p_proj.y < 1.0f + padding);
    if (!visible) {
        radius_out = 0.0f;
        return false;
    }
    const float sx = expf(lscales[3 * idx]), sy = expf(lscales[3 * idx + 1]), sz = expf(lscales[3 * idx + 2]);
    float4 q = {rots[4 * idx], rots[4 * idx + 1], rots[4 * idx + 2], rots[4 * idx + 3]};
    const float rn = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (rn > 0.f) {
        q.x = q.x / rn; q.y = q.y / rn; q.z = q.z / rn; q.w = q.w / rn;
    } else {
        q = {1.f, 0.f, 0.f, 0.f};
    }
    float cov3D[6];
    cov3d_from_scale_rot(sx, sy, sz, 1.f, q, cov3D);
    float3 cov = ewa_cov2d(p_orig, fx, fy, tanx, tany, cov3D, view);
    cov.x = dilate_max(cov.x);
    cov.z = dilate_max(cov.z);
    const float det = (cov.x * cov.z - cov.y * cov.y);
    if (det <= 0.0f) {
        radius_out = 0.0f;
        return true;
    }
    const float mid = 0.5f * (cov.x + cov.z);
    const float disc = fmaxf(0.1f, mid * mid - det);
    const float root = sqrtf(disc);
    const float lambda1 = mid + root;
    const float lambda2 = mid - root;
    radius_out = 3.f * sqrtf(fmaxf(lambda1, lambda2));
    return true;
}

// Phase 1 of compute_radius_kernel_v2.cu:231-353: every node's visibility,
// radius and NDC depth.  Each node's radius is a pure function of the node,
// so computing all of them first and applying the tree rule in phase 2 gives
// the same mask as the reference's lazily computed ancestor radii.
__global__ void visibility_phase1(int P, const float* __restrict__ means, const float* __restrict__ lscales,
                                  const float* __restrict__ rots, const float* __restrict__ proj,
                                  const float* __restrict__ view, float fx, float fy, float tanx, float tany,
                                  float padding, uint8_t* __restrict__ mask, float* __restrict__ radius2d,
                                  float* __restrict__ depth)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    float r = 0.f, d = 0.f;
    const bool vis = vis_radius_point(idx, means, lscales, rots, proj, view, fx, fy, tanx, tany, padding, d, r);
    depth[idx] = d;
    radius2d[idx] = r;
    mask[idx] = vis ? 1 : 0;  // phase 2 turns this into the keep decision
}

// Phase 2: the LoD keep rule (compute_radius_kernel_v2.cu:281-352).
__global__ void visibility_phase2(int P, const int32_t* __restrict__ node_index, const int32_t* __restrict__ anc,
                                  int L, float radius_max, float radius_filter, uint8_t* __restrict__ mask,
                                  const float* __restrict__ radius2d)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    if (!mask[idx]) return;
    const float r = radius2d[idx];
    bool keep = true;
    if (node_index[idx] != -1) {
        keep = r <= radius_max;
    } else {
        const int32_t* row = anc + (size_t)idx * L;
        for (int l = 0; l < L; ++l) {
            const int32_t a = __ldg(row + l);
            if (a < 0) break;
            if (a == idx || a >= P) continue;  // (an id past the node table is not a node)
            if (__ldg(node_index + a) == -1) continue;
            const float ar = radius2d[a];
            if (ar > 0.f && ar <= radius_max) {
                keep = false;
                break;
            }
        }
    }
    if (keep && radius_filter > 0.0f && r > radius_filter) keep = false;
    mask[idx] = keep ? 1 : 0;
}

}  // namespace

void launch_preprocess(const PreParams& p, const GeomState& g, int* radii, cudaStream_t s)
{
    if (p.P <= 0) return;
    const uint32_t nch = (uint32_t)((p.P + kThreads - 1) / kThreads);
    preprocess_cull_kernel<<<min(nch, resident_ctas(preprocess_cull_kernel, kThreads)), kThreads, 0, s>>>(
        p, g, radii);
    preprocess_full_kernel<<<resident_ctas(preprocess_full_kernel, kThreads), kThreads, 0, s>>>(p, g, radii);
    chunk_scan_kernel<<<1, 1024, 0, s>>>(g.chunk_counts, nch, g.total);
    compact_visible_kernel<<<nch, kThreads, 0, s>>>(p.P, g.tiles, g.grec, g.chunk_counts, g.sort_ids_b,
                                                    g.depth_key);
    note_launches(4);
}

void launch_pack_gaussians(int P, const float* means, const float* opac, const float* scales, const float* rots,
                           float4* packed, cudaStream_t s)
{
    if (P <= 0) return;
    const int blocks = (int)min((P + 255) / 256, 148 * 8);
    pack_gaussians_kernel<<<blocks, 256, 0, s>>>(P, means, opac, scales, rots, packed);
    note_launches(1);
}

void launch_compute_radius(int variant, int P, const float* means, const float* scales, const float* rots,
                           const float* view, const float* proj, float fx, float fy, float tanx, float tany,
                           float* radius, cudaStream_t s)
{
    if (P <= 0) return;
    compute_radius_kernel<<<(P + 255) / 256, 256, 0, s>>>(variant, P, means, scales, rots, view, proj, fx, fy,
                                                           tanx, tany, radius);
    note_launches(1);
}

void launch_mark_visible(int P, const float* means, const float* view, uint8_t* present, cudaStream_t s)
{
    if (P <= 0) return;
    mark_visible_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, means, view, present);
    note_launches(1);
}

void launch_visibility_radius(int P, const float* means, const float* lscales, const float* rots,
                              const float* proj, const float* view, const int32_t* node_index,
                              const int32_t* ancestors, int L, float fx, float fy, float tanx, float tany,
                              float padding, float radius_max, float radius_filter, uint8_t* mask, float* radius2d,
                              float* depth, cudaStream_t s)
{
    if (P <= 0) return;
    visibility_phase1<<<(P + 255) / 256, 256, 0, s>>>(P, means, lscales, rots, proj, view, fx, fy, tanx, tany,
                                                       padding, mask, radius2d, depth);
    visibility_phase2<<<(P + 255) / 256, 256, 0, s>>>(P, node_index, ancestors, L, radius_max, radius_filter,
                                                       mask, radius2d);
    note_launches(2);
}

}  // namespace fgs
