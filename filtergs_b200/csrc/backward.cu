// Per-Gaussian backward: 2D-covariance, projection, SH and scale/rotation
// gradients in one kernel (antialias/cuda_rasterizer/backward.cu:20-396,
// where computeCov2DCUDA and preprocessCUDA are two launches).
//
// The 3D covariance is recomputed from scale/rotation (it is a pure function
// of them) instead of being kept in the geometry buffer.  Every output row is
// written, zeros for Gaussians the forward culled, so the caller needs no
// zero-initialisation.
//
// mode FGS_BACKWARD_REF_COMPAT reproduces the reference: the 2D covariance is
// dilated by +0.3 (backward.cu:197-199) whatever the forward did, and
// 1/(det^2 + 1e-7) is used.  FGS_BACKWARD_CONSISTENT differentiates the
// forward as computed: max(., 0.3) dilation only when use_filter, with a zero
// gradient for a clamped diagonal entry, exact 1/det^2, and the t.z
// dependence of a clamped t.x / t.y.
#include <algorithm>

#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

__device__ __forceinline__ float3 dnormvdv(float3 v, float3 dv)
{
    const float sum2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const float invsum32 = 1.0f / sqrtf(sum2 * sum2 * sum2);
    float3 r;
    r.x = ((+sum2 - v.x * v.x) * dv.x - v.y * v.x * dv.y - v.z * v.x * dv.z) * invsum32;
    r.y = (-v.x * v.y * dv.x + (sum2 - v.y * v.y) * dv.y - v.z * v.y * dv.z) * invsum32;
    r.z = (-v.x * v.z * dv.x - v.y * v.z * dv.y + (sum2 - v.z * v.z) * dv.z) * invsum32;
    return r;
}

// backward.cu:20-139 for one Gaussian; shrow / dsh are its [M][3] rows (added to
// dsh instead of stored when kAccum; vec: both rows 16-byte aligned, M*3 % 4 == 0).
// dL/dsh depends only on the direction, so it is written before the SH row is
// read: the two 48-float sets are never live at the same time.
template <bool kAccum>
__device__ __forceinline__ float3 sh_backward(int deg, const float* __restrict__ shrow, float3 pos, float3 campos,
                                              uint8_t clamp_bits, float3 dcol, float* __restrict__ dsh, int M,
                                              bool vec)
{
    const float3 dir_orig = {pos.x - campos.x, pos.y - campos.y, pos.z - campos.z};
    const float len = sqrtf(dir_orig.x * dir_orig.x + dir_orig.y * dir_orig.y + dir_orig.z * dir_orig.z);
    const float x = dir_orig.x / len, y = dir_orig.y / len, z = dir_orig.z / len;
    const float d[3] = {(clamp_bits & 1) ? 0.f : dcol.x, (clamp_bits & 2) ? 0.f : dcol.y,
                        (clamp_bits & 4) ? 0.f : dcol.z};
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    // basis values (dL/dsh[i][c] = B[i] * d[c])
    float B[16];
    B[0] = kSH_C0;
    B[1] = -kSH_C1 * y;
    B[2] = kSH_C1 * z;
    B[3] = -kSH_C1 * x;
    B[4] = kSH_C2_0 * xy;
    B[5] = kSH_C2_1 * yz;
    B[6] = kSH_C2_2 * (2.f * zz - xx - yy);
    B[7] = kSH_C2_3 * xz;
    B[8] = kSH_C2_4 * (xx - yy);
    B[9] = kSH_C3_0 * y * (3.f * xx - yy);
    B[10] = kSH_C3_1 * xy * z;
    B[11] = kSH_C3_2 * y * (4.f * zz - xx - yy);
    B[12] = kSH_C3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
    B[13] = kSH_C3_4 * x * (4.f * zz - xx - yy);
    B[14] = kSH_C3_5 * z * (xx - yy);
    B[15] = kSH_C3_6 * x * (xx - 3.f * yy);
    const int ncoef = (deg + 1) * (deg + 1);
    const int nfl = M * 3;
#define FGS_DSH(f) (((f) / 3 < ncoef) ? B[(f) / 3] * d[(f) % 3] : 0.f)
    if (vec) {
        float4* d4 = reinterpret_cast<float4*>(dsh);
#pragma unroll
        for (int v = 0; v < 12; v++)
            if (4 * v < nfl) {
                float4 o = make_float4(FGS_DSH(4 * v), FGS_DSH(4 * v + 1), FGS_DSH(4 * v + 2), FGS_DSH(4 * v + 3));
                if (kAccum) {
                    const float4 a = d4[v];
                    o.x += a.x; o.y += a.y; o.z += a.z; o.w += a.w;
                }
                d4[v] = o;
            }
    } else {
#pragma unroll
        for (int f = 0; f < 48; f++)
            if (f < nfl) {
                if (kAccum) dsh[f] += FGS_DSH(f);
                else dsh[f] = FGS_DSH(f);
            }
    }
#undef FGS_DSH
    if (!kAccum)
        for (int f = 48; f < nfl; f++) dsh[f] = 0.f;
    if (deg == 0) return make_float3(0.f, 0.f, 0.f);

    // dRGB/ddir (backward.cu:59-124 expression order) from the SH row
    float sh[48];
    const int nf = min(48, nfl);
    if (vec) {
        const float4* r4 = reinterpret_cast<const float4*>(shrow);
#pragma unroll
        for (int v = 0; v < 12; v++)
            if (4 * v < nf) {
                const float4 q = __ldg(r4 + v);
                sh[4 * v] = q.x; sh[4 * v + 1] = q.y; sh[4 * v + 2] = q.z; sh[4 * v + 3] = q.w;
            }
    } else {
#pragma unroll
        for (int f = 0; f < 48; f++)
            if (f < nf) sh[f] = __ldg(shrow + f);
    }
    float dx[3], dy[3], dz[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        dx[c] = -kSH_C1 * sh[9 + c];
        dy[c] = -kSH_C1 * sh[3 + c];
        dz[c] = kSH_C1 * sh[6 + c];
    }
    if (deg > 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dx[c] += kSH_C2_0 * y * sh[12 + c] + kSH_C2_2 * 2.f * -x * sh[18 + c] + kSH_C2_3 * z * sh[21 + c] +
                     kSH_C2_4 * 2.f * x * sh[24 + c];
            dy[c] += kSH_C2_0 * x * sh[12 + c] + kSH_C2_1 * z * sh[15 + c] + kSH_C2_2 * 2.f * -y * sh[18 + c] +
                     kSH_C2_4 * 2.f * -y * sh[24 + c];
            dz[c] += kSH_C2_1 * y * sh[15 + c] + kSH_C2_2 * 2.f * 2.f * z * sh[18 + c] + kSH_C2_3 * x * sh[21 + c];
        }
        if (deg > 2) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                dx[c] += (kSH_C3_0 * sh[27 + c] * 3.f * 2.f * xy + kSH_C3_1 * sh[30 + c] * yz +
                          kSH_C3_2 * sh[33 + c] * -2.f * xy + kSH_C3_3 * sh[36 + c] * -3.f * 2.f * xz +
                          kSH_C3_4 * sh[39 + c] * (-3.f * xx + 4.f * zz - yy) + kSH_C3_5 * sh[42 + c] * 2.f * xz +
                          kSH_C3_6 * sh[45 + c] * 3.f * (xx - yy));
                dy[c] += (kSH_C3_0 * sh[27 + c] * 3.f * (xx - yy) + kSH_C3_1 * sh[30 + c] * xz +
                          kSH_C3_2 * sh[33 + c] * (-3.f * yy + 4.f * zz - xx) +
                          kSH_C3_3 * sh[36 + c] * -3.f * 2.f * yz + kSH_C3_4 * sh[39 + c] * -2.f * xy +
                          kSH_C3_5 * sh[42 + c] * -2.f * yz + kSH_C3_6 * sh[45 + c] * -3.f * 2.f * xy);
                dz[c] += (kSH_C3_1 * sh[30 + c] * xy + kSH_C3_2 * sh[33 + c] * 4.f * 2.f * yz +
                          kSH_C3_3 * sh[36 + c] * 3.f * (2.f * zz - xx - yy) + kSH_C3_4 * sh[39 + c] * 4.f * 2.f * xz +
                          kSH_C3_5 * sh[42 + c] * (xx - yy));
            }
        }
    }
    const float3 ddir = {dx[0] * d[0] + dx[1] * d[1] + dx[2] * d[2], dy[0] * d[0] + dy[1] * d[1] + dy[2] * d[2],
                         dz[0] * d[0] + dz[1] * d[1] + dz[2] * d[2]};
    return dnormvdv(dir_orig, ddir);
}

// Screen-space gradients of the visible Gaussians: the sum of each Gaussian's
// per-pair gradients (pgrad rows at its emission indices, its tiles row-major).
// Gaussians are taken in depth rank j, whose pairs are the contiguous rows
// [pair_off[j], pair_off[j + 1]) (the last ends at K), so a warp reads its next
// Gaussian's row range while it sums the current one.  One warp per Gaussian:
// lane l takes rows l, l+32, ... (coalesced 36-byte rows, 128 rows in flight per
// round trip, so a splat over thousands of tiles does not stall the kernel) and a
// fixed shuffle tree adds them, 32 rows at a time in emission order -- the same
// sum on every run.  Row layout: dcolor r,g,b | dmean2D x,y | dconic x,y,w |
// dopacity.
__global__ void __launch_bounds__(256)
    pair_grad_gather_kernel(const uint32_t* __restrict__ visible_ids, const unsigned long long* __restrict__ totals,
                            const uint32_t* __restrict__ pair_off, const float* __restrict__ pgrad,
                            float* __restrict__ dmean2D, float* __restrict__ dconic, float* __restrict__ dcolor,
                            float* __restrict__ dopac, float* __restrict__ dens_grad, int* __restrict__ dens_count,
                            uint8_t* __restrict__ dens_flag)
{
    const uint32_t K = (uint32_t)totals[0], V = (uint32_t)totals[1];
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    auto range = [&](uint32_t jj, uint32_t& e0, uint32_t& e1, int& idx) {
        e0 = __ldg(pair_off + jj);
        e1 = jj + 1 < V ? __ldg(pair_off + jj + 1) : K;
        idx = (int)__ldg(visible_ids + jj);
    };
    uint32_t e0 = 0, e1 = 0;
    int idx = 0;
    if (j < V) range(j, e0, e1, idx);
    while (j < V) {
        const uint32_t jn = j + nwarps;
        uint32_t n0 = 0, n1 = 0;
        int nidx = 0;
        if (jn < V) range(jn, n0, n1, nidx);  // the next Gaussian's rows, in flight meanwhile
        const uint32_t ne = e1 - e0;
        float acc = 0.f;  // lanes 2q and 2q+1: component q
        for (uint32_t k = 0; k < ne; k += 128) {
            float v[4][9];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t r = k + 32 * u + lane;
                const float* src = pgrad + (size_t)(e0 + r) * 9;
#pragma unroll
                for (int q = 0; q < 9; q++) v[u][q] = r < ne ? __ldg(src + q) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (k + 32 * u < ne) acc += warp_transpose_sum9(v[u]);
        }
        if (dens_grad) {
            // densification statistics (LoG/model/counter.py): |dL/dmean2D[:2]| and visibility
            const float gx = __shfl_sync(0xffffffffu, acc, 6), gy = __shfl_sync(0xffffffffu, acc, 8);
            if (lane == 0) {
                dens_grad[idx] += sqrtf(gx * gx + gy * gy);
                dens_count[idx] += 1;
                dens_flag[idx] = 1;
            }
        }
        if (lane < 18 && !(lane & 1)) {
            const int q = lane >> 1;
            float* dst = q < 3 ? dcolor + 3 * idx + q
                       : q < 5 ? dmean2D + 3 * idx + (q - 3)
                       : q == 7 ? dconic + 4 * idx + 3
                       : q < 8 ? dconic + 4 * idx + (q - 5)
                               : dopac + idx;
            *dst = acc;
        }
        j = jn;
        e0 = n0;
        e1 = n1;
        idx = nidx;
    }
}

// kAccum: add this view's gradients into dense buffers shared by several views
// (views run one after another on a stream, so each row has one writer at a
// time) and fold the view's opacity gradient into shared_dopac.
template <bool kAccum>
__global__ void __launch_bounds__(256)
    preprocess_bwd_kernel(PreParams p, const uint32_t* __restrict__ visible_ids,
                          const unsigned long long* __restrict__ visible_count, float* __restrict__ dmean2D,
                          const float* __restrict__ dconic, float* __restrict__ dopac, float* __restrict__ dmean3D,
                          float* __restrict__ dcov3D,
                          float* __restrict__ dscale, float* __restrict__ drot, int consistent,
                          float* __restrict__ shared_dopac, bool sh_follows)
{
    // The forward's depth ordering put the V visible Gaussians first; culled
    // rows were zero-filled by the launcher.
    const uint32_t V = (uint32_t)*visible_count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < V; j += gridDim.x * blockDim.x) {
    const int idx = (int)visible_ids[j];
    float3 dm = {0.f, 0.f, 0.f};
    float dc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    {
        const float3 mean = {p.means[3 * idx], p.means[3 * idx + 1], p.means[3 * idx + 2]};
        float cov3D[6];
        if (p.cov3D) {
#pragma unroll
            for (int k = 0; k < 6; k++) cov3D[k] = p.cov3D[6 * (size_t)idx + k];
        } else {
            const float4 q = {p.rots[4 * idx], p.rots[4 * idx + 1], p.rots[4 * idx + 2], p.rots[4 * idx + 3]};
            cov3d_from_scale_rot(p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2], p.scale_mod, q,
                                 cov3D);
        }
        if (p.filter3d > 0.f) {
            const float3 pv = xform_point4x3(mean, p.view);
            const float sf = p.filter3d * pv.z / p.fx;
            const float v = sf * sf;
            cov3D[0] += v; cov3D[3] += v; cov3D[5] += v;
        }
        const float3 dL_dconic = {dconic[4 * idx], dconic[4 * idx + 1], dconic[4 * idx + 3]};
        Ewa e;
        const float3 c2 = ewa_cov2d(mean, p.fx, p.fy, p.tanx, p.tany, cov3D, p.view, &e);
        float a, b = c2.y, c;
        float mask_a = 1.f, mask_c = 1.f;
        if (consistent) {
            if (p.use_filter) {
                a = dilate_max(c2.x);
                c = dilate_max(c2.z);
                if (!((double)c2.x > 0.3)) mask_a = 0.f;
                if (!((double)c2.z > 0.3)) mask_c = 0.f;
            } else {
                a = c2.x;
                c = c2.z;
            }
        } else {
            a = dilate_add(c2.x);
            c = dilate_add(c2.z);
        }
        const float denom = a * c - b * b;
        float dL_da = 0, dL_db = 0, dL_dc = 0;
        const float denom2inv = consistent ? 1.0f / (denom * denom) : 1.0f / ((denom * denom) + 0.0000001f);
        const M3& T = e.T;
        if (denom2inv != 0) {
            dL_da = denom2inv * (-c * c * dL_dconic.x + 2 * b * c * dL_dconic.y + (denom - a * c) * dL_dconic.z);
            dL_dc = denom2inv * (-a * a * dL_dconic.z + 2 * a * b * dL_dconic.y + (denom - a * c) * dL_dconic.x);
            dL_db = denom2inv * 2 * (b * c * dL_dconic.x - (denom + 2 * b * b) * dL_dconic.y + a * b * dL_dconic.z);
            dL_da *= mask_a;
            dL_dc *= mask_c;
            dc[0] = (T.m[0][0] * T.m[0][0] * dL_da + T.m[0][0] * T.m[1][0] * dL_db + T.m[1][0] * T.m[1][0] * dL_dc);
            dc[3] = (T.m[0][1] * T.m[0][1] * dL_da + T.m[0][1] * T.m[1][1] * dL_db + T.m[1][1] * T.m[1][1] * dL_dc);
            dc[5] = (T.m[0][2] * T.m[0][2] * dL_da + T.m[0][2] * T.m[1][2] * dL_db + T.m[1][2] * T.m[1][2] * dL_dc);
            dc[1] = 2 * T.m[0][0] * T.m[0][1] * dL_da + (T.m[0][0] * T.m[1][1] + T.m[0][1] * T.m[1][0]) * dL_db +
                    2 * T.m[1][0] * T.m[1][1] * dL_dc;
            dc[2] = 2 * T.m[0][0] * T.m[0][2] * dL_da + (T.m[0][0] * T.m[1][2] + T.m[0][2] * T.m[1][0]) * dL_db +
                    2 * T.m[1][0] * T.m[1][2] * dL_dc;
            dc[4] = 2 * T.m[0][2] * T.m[0][1] * dL_da + (T.m[0][1] * T.m[1][2] + T.m[0][2] * T.m[1][1]) * dL_db +
                    2 * T.m[1][1] * T.m[1][2] * dL_dc;
        }
        // Vrk[c][r]
        const float V00 = cov3D[0], V01 = cov3D[1], V02 = cov3D[2], V11 = cov3D[3], V12 = cov3D[4], V22 = cov3D[5];
        const float V10 = V01, V20 = V02, V21 = V12;
        const float dL_dT00 = 2 * (T.m[0][0] * V00 + T.m[0][1] * V01 + T.m[0][2] * V02) * dL_da +
                              (T.m[1][0] * V00 + T.m[1][1] * V01 + T.m[1][2] * V02) * dL_db;
        const float dL_dT01 = 2 * (T.m[0][0] * V10 + T.m[0][1] * V11 + T.m[0][2] * V12) * dL_da +
                              (T.m[1][0] * V10 + T.m[1][1] * V11 + T.m[1][2] * V12) * dL_db;
        const float dL_dT02 = 2 * (T.m[0][0] * V20 + T.m[0][1] * V21 + T.m[0][2] * V22) * dL_da +
                              (T.m[1][0] * V20 + T.m[1][1] * V21 + T.m[1][2] * V22) * dL_db;
        const float dL_dT10 = 2 * (T.m[1][0] * V00 + T.m[1][1] * V01 + T.m[1][2] * V02) * dL_dc +
                              (T.m[0][0] * V00 + T.m[0][1] * V01 + T.m[0][2] * V02) * dL_db;
        const float dL_dT11 = 2 * (T.m[1][0] * V10 + T.m[1][1] * V11 + T.m[1][2] * V12) * dL_dc +
                              (T.m[0][0] * V10 + T.m[0][1] * V11 + T.m[0][2] * V12) * dL_db;
        const float dL_dT12 = 2 * (T.m[1][0] * V20 + T.m[1][1] * V21 + T.m[1][2] * V22) * dL_dc +
                              (T.m[0][0] * V20 + T.m[0][1] * V21 + T.m[0][2] * V22) * dL_db;
        // W[c][r] = view[c + 4r]
        const float* v = p.view;
        const float dL_dJ00 = v[0] * dL_dT00 + v[4] * dL_dT01 + v[8] * dL_dT02;
        const float dL_dJ02 = v[2] * dL_dT00 + v[6] * dL_dT01 + v[10] * dL_dT02;
        const float dL_dJ11 = v[1] * dL_dT10 + v[5] * dL_dT11 + v[9] * dL_dT12;
        const float dL_dJ12 = v[2] * dL_dT10 + v[6] * dL_dT11 + v[10] * dL_dT12;
        const float tz = 1.f / e.tz;
        const float tz2 = tz * tz;
        const float tz3 = tz2 * tz;
        const float x_grad_mul = e.xclamp ? 0 : 1;
        const float y_grad_mul = e.yclamp ? 0 : 1;
        const float dL_dtx = x_grad_mul * -p.fx * tz2 * dL_dJ02;
        const float dL_dty = y_grad_mul * -p.fy * tz2 * dL_dJ12;
        float dL_dtz = -p.fx * tz2 * dL_dJ00 - p.fy * tz2 * dL_dJ11 + (2 * p.fx * e.tx) * tz3 * dL_dJ02 +
                       (2 * p.fy * e.ty) * tz3 * dL_dJ12;
        if (consistent) {
            const float limx = 1.3f * p.tanx, limy = 1.3f * p.tany;
            if (e.xclamp) dL_dtz += (-p.fx * tz2 * dL_dJ02) * (e.txtz < 0 ? -limx : limx);
            if (e.yclamp) dL_dtz += (-p.fy * tz2 * dL_dJ12) * (e.tytz < 0 ? -limy : limy);
        }
        // transformVec4x3Transpose
        dm.x = v[0] * dL_dtx + v[1] * dL_dty + v[2] * dL_dtz;
        dm.y = v[4] * dL_dtx + v[5] * dL_dty + v[6] * dL_dtz;
        dm.z = v[8] * dL_dtx + v[9] * dL_dty + v[10] * dL_dtz;

        // backward.cu:370-387: screen-space mean gradient through the projection
        const float* pr = p.proj;
        const float4 m_hom = xform_point4x4(mean, pr);
        const float m_w = 1.0f / (m_hom.w + 0.0000001f);
        const float mul1 = (pr[0] * mean.x + pr[4] * mean.y + pr[8] * mean.z + pr[12]) * m_w * m_w;
        const float mul2 = (pr[1] * mean.x + pr[5] * mean.y + pr[9] * mean.z + pr[13]) * m_w * m_w;
        const float g2x = dmean2D[3 * idx], g2y = dmean2D[3 * idx + 1];
        dm.x += (pr[0] * m_w - pr[3] * mul1) * g2x + (pr[1] * m_w - pr[3] * mul2) * g2y;
        dm.y += (pr[4] * m_w - pr[7] * mul1) * g2x + (pr[5] * m_w - pr[7] * mul2) * g2y;
        dm.z += (pr[8] * m_w - pr[11] * mul1) * g2x + (pr[9] * m_w - pr[11] * mul2) * g2y;

        if (p.scales && dscale) {
            // backward.cu:278-341 (gradient w.r.t. the quaternion as given)
            const float r = p.rots[4 * idx], x = p.rots[4 * idx + 1], y = p.rots[4 * idx + 2], z = p.rots[4 * idx + 3];
            const M3 R = m3_cols(1.f - 2.f * (y * y + z * z), 2.f * (x * y - r * z), 2.f * (x * z + r * y),
                                 2.f * (x * y + r * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - r * x),
                                 2.f * (x * z - r * y), 2.f * (y * z + r * x), 1.f - 2.f * (x * x + y * y));
            const float s[3] = {p.scale_mod * p.scales[3 * idx], p.scale_mod * p.scales[3 * idx + 1],
                                p.scale_mod * p.scales[3 * idx + 2]};
            M3 S = m3_cols(1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f);
            S.m[0][0] = s[0]; S.m[1][1] = s[1]; S.m[2][2] = s[2];
            const M3 M = m3_mul(S, R);
            const M3 dSig = m3_cols(dc[0], 0.5f * dc[1], 0.5f * dc[2], 0.5f * dc[1], dc[3], 0.5f * dc[4], 0.5f * dc[2],
                                    0.5f * dc[4], dc[5]);
            M3 M2;
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int rr = 0; rr < 3; rr++) M2.m[cc][rr] = 2.0f * M.m[cc][rr];
            const M3 dM = m3_mul(M2, dSig);
            const M3 Rt = m3_t(R);
            M3 dMt = m3_t(dM);
            float* ds = dscale + 3 * (size_t)idx;
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
            {
                const float v = Rt.m[cc][0] * dMt.m[cc][0] + Rt.m[cc][1] * dMt.m[cc][1] + Rt.m[cc][2] * dMt.m[cc][2];
                if (kAccum) ds[cc] += v;
                else ds[cc] = v;
            }
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int rr = 0; rr < 3; rr++) dMt.m[cc][rr] *= s[cc];
            float4 dq;
            dq.x = 2 * z * (dMt.m[0][1] - dMt.m[1][0]) + 2 * y * (dMt.m[2][0] - dMt.m[0][2]) +
                   2 * x * (dMt.m[1][2] - dMt.m[2][1]);
            dq.y = 2 * y * (dMt.m[1][0] + dMt.m[0][1]) + 2 * z * (dMt.m[2][0] + dMt.m[0][2]) +
                   2 * r * (dMt.m[1][2] - dMt.m[2][1]) - 4 * x * (dMt.m[2][2] + dMt.m[1][1]);
            dq.z = 2 * x * (dMt.m[1][0] + dMt.m[0][1]) + 2 * r * (dMt.m[2][0] - dMt.m[0][2]) +
                   2 * z * (dMt.m[1][2] + dMt.m[2][1]) - 4 * y * (dMt.m[2][2] + dMt.m[0][0]);
            dq.w = 2 * r * (dMt.m[0][1] - dMt.m[1][0]) + 2 * x * (dMt.m[2][0] + dMt.m[0][2]) +
                   2 * y * (dMt.m[1][2] + dMt.m[2][1]) - 4 * z * (dMt.m[1][1] + dMt.m[0][0]);
            float* dr = drot + 4 * (size_t)idx;
            if (kAccum) {
                dr[0] += dq.x; dr[1] += dq.y; dr[2] += dq.z; dr[3] += dq.w;
            } else {
                dr[0] = dq.x; dr[1] = dq.y; dr[2] = dq.z; dr[3] = dq.w;
            }
        }
        const bool floor_mask = consistent && p.opac && p.opac[idx] < 1e-6f;
        if (kAccum) {
            if (!floor_mask) shared_dopac[idx] += dopac[idx];
        } else if (floor_mask) {
            dopac[idx] = 0.f;
        }
    }
    if (kAccum && sh_follows) {
        // the SH pass adds its term and then accumulates the view's total (the same
        // sum, in the same order, as the plain backward of this view)
        dmean2D[3 * idx] = dm.x;
        dmean2D[3 * idx + 1] = dm.y;
        dmean2D[3 * idx + 2] = dm.z;
#pragma unroll
        for (int k = 0; k < 6; k++) dcov3D[6 * (size_t)idx + k] += dc[k];
    } else if (kAccum) {
        dmean3D[3 * idx] += dm.x;
        dmean3D[3 * idx + 1] += dm.y;
        dmean3D[3 * idx + 2] += dm.z;
#pragma unroll
        for (int k = 0; k < 6; k++) dcov3D[6 * (size_t)idx + k] += dc[k];
    } else {
        dmean3D[3 * idx] = dm.x;
        dmean3D[3 * idx + 1] = dm.y;
        dmean3D[3 * idx + 2] = dm.z;
#pragma unroll
        for (int k = 0; k < 6; k++) dcov3D[6 * (size_t)idx + k] = dc[k];
    }
    }
}

// SH part of the per-Gaussian backward as its own pass over the visible ids
// (after preprocess_bwd_kernel on the same stream): dL/dsh and the SH term of
// dL/dmean, added to the row preprocess_bwd_kernel wrote.  Kept apart so that
// neither kernel holds the 48-float SH rows next to the covariance chain.
template <bool kAccum>
__global__ void __launch_bounds__(256, 3)
    sh_bwd_kernel(PreParams p, const uint32_t* __restrict__ visible_ids,
                  const unsigned long long* __restrict__ visible_count, const uint8_t* __restrict__ clamped,
                  const float* __restrict__ dcolor, const float* __restrict__ dm_geo, float* __restrict__ dmean3D,
                  float* __restrict__ dsh)
{
    const uint32_t V = (uint32_t)*visible_count;
    const bool vec = p.aligned && ((p.M * 3) & 3) == 0;
    const float3 cam = {p.campos[0], p.campos[1], p.campos[2]};
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < V; j += gridDim.x * blockDim.x) {
        const int idx = (int)visible_ids[j];
        const float3 mean = {p.means[3 * idx], p.means[3 * idx + 1], p.means[3 * idx + 2]};
        const float3 dcol = {dcolor[3 * idx], dcolor[3 * idx + 1], dcolor[3 * idx + 2]};
        const float3 dmd = sh_backward<kAccum>(p.D, p.shs + (size_t)idx * p.M * 3, mean, cam, clamped[idx], dcol,
                                               dsh + (size_t)idx * p.M * 3, p.M, vec);
        if (kAccum) {  // this view's total, then into the shared sum
            dmean3D[3 * idx] += dm_geo[3 * idx] + dmd.x;
            dmean3D[3 * idx + 1] += dm_geo[3 * idx + 1] + dmd.y;
            dmean3D[3 * idx + 2] += dm_geo[3 * idx + 2] + dmd.z;
        } else {
            dmean3D[3 * idx] += dmd.x;
            dmean3D[3 * idx + 1] += dmd.y;
            dmean3D[3 * idx + 2] += dmd.z;
        }
    }
}

}  // namespace

void launch_preprocess_bwd(const PreParams& p, const GeomState& g, const float* pgrad, float* dmean2D, float* dconic,
                           float* dcolor, float* dopac, float* dmean3D, float* dcov3D, float* dsh, float* dscale,
                           float* drot, int consistent, cudaStream_t s, bool accumulate, float* shared_dopac,
                           const DensifyStats* dens)
{
    if (p.P <= 0) return;
    const size_t P = (size_t)p.P;
    if (!accumulate) {
        // Dense outputs: culled rows are zero, written here at copy-engine speed.
        cudaMemsetAsync(dmean3D, 0, sizeof(float) * 3 * P, s);
        cudaMemsetAsync(dcov3D, 0, sizeof(float) * 6 * P, s);
        if (dsh) cudaMemsetAsync(dsh, 0, sizeof(float) * 3 * (size_t)p.M * P, s);
        if (dscale) cudaMemsetAsync(dscale, 0, sizeof(float) * 3 * P, s);
        if (drot) cudaMemsetAsync(drot, 0, sizeof(float) * 4 * P, s);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = (int)std::min<size_t>((P + 255) / 256, (size_t)sms * 8);
    const bool sh = p.shs && dsh;
    pair_grad_gather_kernel<<<blocks, 256, 0, s>>>(g.sort_ids_b, g.total, g.pair_off, pgrad, dmean2D, dconic,
                                                   dcolor, dopac, dens ? dens->grad_sum : nullptr,
                                                   dens ? dens->count : nullptr, dens ? dens->flag : nullptr);
    if (accumulate) {
        preprocess_bwd_kernel<true><<<blocks, 256, 0, s>>>(p, g.sort_ids_b, g.total + 1, dmean2D, dconic, dopac,
                                                           dmean3D, dcov3D, dscale, drot, consistent, shared_dopac, sh);
        if (sh)
            sh_bwd_kernel<true><<<blocks, 256, 0, s>>>(p, g.sort_ids_b, g.total + 1, g.clamped, dcolor, dmean2D,
                                                       dmean3D, dsh);
    } else {
        preprocess_bwd_kernel<false><<<blocks, 256, 0, s>>>(p, g.sort_ids_b, g.total + 1, dmean2D, dconic, dopac,
                                                            dmean3D, dcov3D, dscale, drot, consistent, nullptr, sh);
        if (sh)
            sh_bwd_kernel<false><<<blocks, 256, 0, s>>>(p, g.sort_ids_b, g.total + 1, g.clamped, dcolor, nullptr,
                                                        dmean3D, dsh);
    }
    note_launches(sh ? 3 : 2);
}

}  // namespace fgs
