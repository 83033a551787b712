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
    // the last product rounded on its own: callers add the result to other terms, and an
    // add fused into it would round differently in different kernels
    r.x = __fmul_rn((+sum2 - v.x * v.x) * dv.x - v.y * v.x * dv.y - v.z * v.x * dv.z, invsum32);
    r.y = __fmul_rn(-v.x * v.y * dv.x + (sum2 - v.y * v.y) * dv.y - v.z * v.y * dv.z, invsum32);
    r.z = __fmul_rn(-v.x * v.z * dv.x - v.y * v.z * dv.y + (sum2 - v.z * v.z) * dv.z, invsum32);
    return r;
}

// SH basis at the unit view direction of a Gaussian at pos seen from campos
// (backward.cu:20-57): dL/dsh[i][c] = B[i] * dL/dcolor[c].
__device__ __forceinline__ void sh_dir(float3 pos, float3 campos, float3& dir_orig, float& x, float& y, float& z)
{
    dir_orig = {pos.x - campos.x, pos.y - campos.y, pos.z - campos.z};
    const float len = sqrtf(dir_orig.x * dir_orig.x + dir_orig.y * dir_orig.y + dir_orig.z * dir_orig.z);
    x = dir_orig.x / len;
    y = dir_orig.y / len;
    z = dir_orig.z / len;
}

__device__ __forceinline__ void sh_basis(float3 pos, float3 campos, float3& dir_orig, float& x, float& y, float& z,
                                         float (&B)[16])
{
    sh_dir(pos, campos, dir_orig, x, y, z);
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
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
}

// dL/dmean3D through the view direction (backward.cu:59-139, the expression
// order of the reference): dRGB/ddir from the SH coefficients sh (deg > 0), dotted
// with the clamp-masked dL/dcolor d, through the normalisation.
__device__ __forceinline__ float3 sh_ddir(int deg, const float (&sh)[48], float x, float y, float z,
                                          const float (&d)[3], float3 dir_orig)
{
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
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

// dL/dsh of float f of an [M][3] row: basis value times masked colour gradient.
__device__ __forceinline__ float sh_dsh(int f, int ncoef, const float (&B)[16], const float (&d)[3])
{
    return (f / 3 < ncoef) ? __fmul_rn(B[f / 3], d[f % 3]) : 0.f;
}

// The SH coefficients of one Gaussian (nf <= 48 floats; vec: 16-byte aligned row).
__device__ __forceinline__ void load_sh_row(const float* __restrict__ shrow, int nf, bool vec, float (&sh)[48])
{
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
}

// Screen-space gradients of the visible Gaussians: the sum of each Gaussian's
// per-pair gradients (pgrad rows at its emission indices, its tiles row-major).
// Gaussians are taken in depth rank j, whose pairs are the contiguous rows
// [pair_off[j], pair_off[j + 1]) (the last ends at K), so a warp reads its next
// Gaussian's row range while it sums the current one.  One warp per Gaussian:
// lane l takes rows l, l+32, ... (coalesced 36-byte rows, 64 rows in flight per
// round trip, so a splat over thousands of tiles does not stall the kernel) and a
// fixed shuffle tree adds them, 32 rows at a time in emission order -- the same
// sum on every run.  Two Gaussians of at most 32 rows each (the common case) share
// one round trip.  Row layout: dcolor r,g,b | dmean2D x,y | dconic x,y,w |
// dopacity.  vis (optional): the view sets vis_bit in vis[idx] for every Gaussian
// it sees.  Compiled for 4 blocks per SM (64 registers; measured faster than the
// compiler's 76 with fewer warps).
__global__ void __launch_bounds__(256, 4)
    pair_grad_gather_kernel(const uint32_t* __restrict__ visible_ids, const unsigned long long* __restrict__ totals,
                            const uint32_t* __restrict__ pair_off, const float* __restrict__ pgrad,
                            float* __restrict__ dmean2D, float* __restrict__ dconic, float* __restrict__ dcolor,
                            float* __restrict__ dopac, uint32_t* __restrict__ vis, uint32_t vis_bit, uint32_t rows)
{
    const uint32_t K = (uint32_t)totals[0], V = (uint32_t)totals[1];
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    // rows past `rows` (a batched view truncated at its pair capacity) were never
    // written: each range is clamped to the buffer
    auto range = [&](uint32_t jj, uint32_t& e0, uint32_t& e1, int& idx) {
        e0 = min(__ldg(pair_off + jj), rows);
        e1 = max(e0, min(jj + 1 < V ? __ldg(pair_off + jj + 1) : K, rows));
        idx = (int)__ldg(visible_ids + jj);
    };
    // sum of rows [e0, e1), component sum9_component(lane) on each lane: 32 rows at a time in
    // emission order, each group through the same shuffle tree, added to 0 in turn
    auto sum_rows = [&](uint32_t e0, uint32_t e1) {
        const uint32_t ne = e1 - e0;
        float acc = 0.f;
        for (uint32_t k = 0; k < ne; k += 64) {
            float v[2][9];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                if (k + 32 * u >= ne) continue;  // (warp-uniform) no rows in this group
                const uint32_t r = k + 32 * u + lane;
                const float* src = pgrad + (size_t)(e0 + r) * 9;
#pragma unroll
                for (int q = 0; q < 9; q++) v[u][q] = r < ne ? __ldg(src + q) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (k + 32 * u < ne) acc += warp_transpose_sum9(v[u]);
        }
        return acc;
    };
    auto store = [&](int idx, float acc) {
        if (vis && lane == 0) atomicOr(vis + idx, vis_bit);  // this view sees Gaussian idx
        const int q = sum9_component(lane);
        if (q < 9 && !(lane & 1)) {
            float* dst = q < 3 ? dcolor + 3 * idx + q
                       : q < 5 ? dmean2D + 3 * idx + (q - 3)
                       : q == 7 ? dconic + 4 * idx + 3
                       : q < 8 ? dconic + 4 * idx + (q - 5)
                               : dopac + idx;
            *dst = acc;
        }
    };
    // Gaussians j and j + nwarps together when both have at most 32 rows (most do:
    // a Gaussian covers ~20 tiles at 1080p), so one round trip brings two row sets
    // while the next pair's ranges are fetched; the sums are the ones sum_rows forms.
    uint32_t a0 = 0, a1 = 0, b0 = 0, b1 = 0;
    int ia = 0, ib = 0;
    if (j < V) range(j, a0, a1, ia);
    if (j + nwarps < V) range(j + nwarps, b0, b1, ib);
    while (j < V) {
        const uint32_t jb = j + nwarps, jc = jb + nwarps, jd = jc + nwarps;
        uint32_t c0 = 0, c1 = 0, d0 = 0, d1 = 0;
        int ic = 0, id = 0;
        if (jb < V && a1 - a0 <= 32 && b1 - b0 <= 32) {
            if (jc < V) range(jc, c0, c1, ic);  // the next pair, in flight meanwhile
            if (jd < V) range(jd, d0, d1, id);
            float va[9], vb[9];
            const float* sa = pgrad + (size_t)(a0 + lane) * 9;
            const float* sb = pgrad + (size_t)(b0 + lane) * 9;
#pragma unroll
            for (int q = 0; q < 9; q++) {
                va[q] = lane < a1 - a0 ? __ldg(sa + q) : 0.f;
                vb[q] = lane < b1 - b0 ? __ldg(sb + q) : 0.f;
            }
            const float ta = warp_transpose_sum9(va), tb = warp_transpose_sum9(vb);
            store(ia, a1 > a0 ? 0.f + ta : 0.f);
            store(ib, b1 > b0 ? 0.f + tb : 0.f);
            j = jc;
            a0 = c0; a1 = c1; ia = ic;
            b0 = d0; b1 = d1; ib = id;
            continue;
        }
        // one Gaussian (long row ranges, or the last one): the next ranges in flight
        if (jc < V) range(jc, c0, c1, ic);
        store(ia, sum_rows(a0, a1));
        j = jb;
        a0 = b0; a1 = b1; ia = ib;
        b0 = c0; b1 = c1; ib = ic;
    }
}

// One view's geometric backward of Gaussian idx (backward.cu:144-396 without the
// SH part): from its screen-space gradients (g2x, g2y of dL/dmean2D, dL/dconic) to
// the geometric dL/dmean3D, dL/dcov3D and, with want_sr, dL/dscale and
// dL/drotation.  floor_mask: the consistent mode gives no opacity gradient to an
// opacity under the 1e-6 floor.
struct GeoGrad {
    float3 dm;
    float dc[6];
    float ds[3];
    float4 dq;
    bool floor_mask;
};

__device__ __forceinline__ void geo_backward(const PreParams& p, int idx, float g2x, float g2y, float3 dL_dconic,
                                             int consistent, bool want_sr, GeoGrad& o)
{
    o.dm = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 6; k++) o.dc[k] = 0.f;
    const float3 mean = {p.means[3 * idx], p.means[3 * idx + 1], p.means[3 * idx + 2]};
    float cov3D[6];
    if (p.cov3D) {
#pragma unroll
        for (int k = 0; k < 6; k++) cov3D[k] = p.cov3D[6 * (size_t)idx + k];
    } else {
        const float4 q = {p.rots[4 * idx], p.rots[4 * idx + 1], p.rots[4 * idx + 2], p.rots[4 * idx + 3]};
        // the forward's cov3D (the reference's backward reads the one its forward stored)
        cov3d_ref(p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2], p.scale_mod, q, cov3D);
    }
    if (p.filter3d > 0.f) {
        const float3 pv = xform_point4x3(mean, p.view);
        const float sf = __fdiv_rn(__fmul_rn(p.filter3d, pv.z), p.fx);
        const float v = __fmul_rn(sf, sf);
        cov3D[0] = __fadd_rn(cov3D[0], v); cov3D[3] = __fadd_rn(cov3D[3], v); cov3D[5] = __fadd_rn(cov3D[5], v);
    }
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
        o.dc[0] = (T.m[0][0] * T.m[0][0] * dL_da + T.m[0][0] * T.m[1][0] * dL_db + T.m[1][0] * T.m[1][0] * dL_dc);
        o.dc[3] = (T.m[0][1] * T.m[0][1] * dL_da + T.m[0][1] * T.m[1][1] * dL_db + T.m[1][1] * T.m[1][1] * dL_dc);
        o.dc[5] = (T.m[0][2] * T.m[0][2] * dL_da + T.m[0][2] * T.m[1][2] * dL_db + T.m[1][2] * T.m[1][2] * dL_dc);
        o.dc[1] = 2 * T.m[0][0] * T.m[0][1] * dL_da + (T.m[0][0] * T.m[1][1] + T.m[0][1] * T.m[1][0]) * dL_db +
                  2 * T.m[1][0] * T.m[1][1] * dL_dc;
        o.dc[2] = 2 * T.m[0][0] * T.m[0][2] * dL_da + (T.m[0][0] * T.m[1][2] + T.m[0][2] * T.m[1][0]) * dL_db +
                  2 * T.m[1][0] * T.m[1][2] * dL_dc;
        o.dc[4] = 2 * T.m[0][2] * T.m[0][1] * dL_da + (T.m[0][1] * T.m[1][2] + T.m[0][2] * T.m[1][1]) * dL_db +
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
    o.dm.x = v[0] * dL_dtx + v[1] * dL_dty + v[2] * dL_dtz;
    o.dm.y = v[4] * dL_dtx + v[5] * dL_dty + v[6] * dL_dtz;
    o.dm.z = v[8] * dL_dtx + v[9] * dL_dty + v[10] * dL_dtz;

    // backward.cu:370-387: screen-space mean gradient through the projection
    const float* pr = p.proj;
    const float4 m_hom = xform_point4x4(mean, pr);
    const float m_w = 1.0f / (m_hom.w + 0.0000001f);
    const float mul1 = (pr[0] * mean.x + pr[4] * mean.y + pr[8] * mean.z + pr[12]) * m_w * m_w;
    const float mul2 = (pr[1] * mean.x + pr[5] * mean.y + pr[9] * mean.z + pr[13]) * m_w * m_w;
    o.dm.x += (pr[0] * m_w - pr[3] * mul1) * g2x + (pr[1] * m_w - pr[3] * mul2) * g2y;
    o.dm.y += (pr[4] * m_w - pr[7] * mul1) * g2x + (pr[5] * m_w - pr[7] * mul2) * g2y;
    o.dm.z += (pr[8] * m_w - pr[11] * mul1) * g2x + (pr[9] * m_w - pr[11] * mul2) * g2y;

    if (want_sr) {
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
        const M3 dSig = m3_cols(o.dc[0], 0.5f * o.dc[1], 0.5f * o.dc[2], 0.5f * o.dc[1], o.dc[3], 0.5f * o.dc[4],
                                0.5f * o.dc[2], 0.5f * o.dc[4], o.dc[5]);
        M3 M2;
#pragma unroll
        for (int cc = 0; cc < 3; cc++)
#pragma unroll
            for (int rr = 0; rr < 3; rr++) M2.m[cc][rr] = 2.0f * M.m[cc][rr];
        const M3 dM = m3_mul(M2, dSig);
        const M3 Rt = m3_t(R);
        M3 dMt = m3_t(dM);
#pragma unroll
        for (int cc = 0; cc < 3; cc++)
            o.ds[cc] = Rt.m[cc][0] * dMt.m[cc][0] + Rt.m[cc][1] * dMt.m[cc][1] + Rt.m[cc][2] * dMt.m[cc][2];
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
        o.dq = dq;
    }
    o.floor_mask = consistent && p.opac && p.opac[idx] < 1e-6f;
}

// ---------------------------------------------------------------- one pass per Gaussian over its views
// The per-Gaussian part of the backward, for one view (the plain path) or many
// (the batched path) with the same code, so that a batch's sums are the plain
// per-view results added in view order, bit for bit.  A thread takes one
// Gaussian of a list of the Gaussians some view saw, walks those views in view
// order, adds each view's whole contribution into registers with explicit
// round-to-nearest adds (no multiply of a per-view term is fused into them) and
// writes the Gaussian's output rows once; the rows of Gaussians no view saw are
// zeroed by the launcher.  No launch per view, no re-reading of shared rows per
// view, and every thread of a warp does a seen Gaussian's work.
//
// list / count: the Gaussians (count[0] of them, any order).  Which views saw
// Gaussian i: vis[(w * P) + i] bit b for view 32 w + b (the batched path, set by
// the views' gathers); with vis null, the one view (the plain path, whose list is
// the view's visible Gaussians: radii > 0, which the reference's backward gates
// every per-Gaussian gradient on, backward.cu:156,367).
__device__ __forceinline__ uint32_t views_of(const uint32_t* __restrict__ vis, int w, int P, int i)
{
    return vis ? vis[(size_t)w * P + i] : 1u;
}

// Geometric part: dL/dopacity, dL/dscale, dL/drotation, dL/dcov3D (optional) and
// each view's geometric dL/dmean3D in its dm_geo row for fold_shdir_kernel (with
// SH), else the dL/dmean3D sum itself.  Densification statistics (optional) as
// densify passes run per view would add them.
__global__ void __launch_bounds__(128, 4)
    fold_geo_kernel(const FoldView* __restrict__ views, FoldView single, int nviews, int P,
                    const uint32_t* __restrict__ list, const unsigned long long* __restrict__ count,
                    const uint32_t* __restrict__ vis, int consistent, bool sh_follows, float* __restrict__ dmean3D,
                    float* __restrict__ dopac_out, float* __restrict__ dcov3D, float* __restrict__ dscale,
                    float* __restrict__ drot, DensifyStats dens)
{
    const int words = (nviews + 31) >> 5;
    const bool want_sr = single.p.scales && dscale;
    const uint32_t n = (uint32_t)*count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = (int)list[j];
        float3 am = {0.f, 0.f, 0.f};
        float adc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float ads[3] = {0.f, 0.f, 0.f};
        float4 adq = {0.f, 0.f, 0.f, 0.f};
        float ado = 0.f;
        float dg = 0.f;
        int seen = 0;
        for (int w = 0; w < words; w++) {
            uint32_t m = views_of(vis, w, P, i);
            while (m) {
                const int v = 32 * w + __ffs(m) - 1;
                m &= m - 1;
                const FoldView& fv = views ? views[v] : single;
                const float g2x = fv.dmean2D[3 * i], g2y = fv.dmean2D[3 * i + 1];
                if (dens.grad_sum) {
                    if (seen == 0) dg = dens.grad_sum[i];
                    dg = __fadd_rn(dg, sqrtf(g2x * g2x + g2y * g2y));
                }
                seen++;
                GeoGrad o;
                geo_backward(fv.p, i, g2x, g2y, {fv.dconic[4 * i], fv.dconic[4 * i + 1], fv.dconic[4 * i + 3]},
                             consistent, want_sr, o);
#pragma unroll
                for (int k = 0; k < 6; k++) adc[k] = __fadd_rn(adc[k], o.dc[k]);
                if (want_sr) {
                    ads[0] = __fadd_rn(ads[0], o.ds[0]);
                    ads[1] = __fadd_rn(ads[1], o.ds[1]);
                    ads[2] = __fadd_rn(ads[2], o.ds[2]);
                    adq.x = __fadd_rn(adq.x, o.dq.x);
                    adq.y = __fadd_rn(adq.y, o.dq.y);
                    adq.z = __fadd_rn(adq.z, o.dq.z);
                    adq.w = __fadd_rn(adq.w, o.dq.w);
                }
                if (!o.floor_mask) ado = __fadd_rn(ado, fv.dopac[i]);
                if (sh_follows) {
                    fv.dm_geo[3 * i] = o.dm.x;
                    fv.dm_geo[3 * i + 1] = o.dm.y;
                    fv.dm_geo[3 * i + 2] = o.dm.z;
                } else {
                    am.x = __fadd_rn(am.x, o.dm.x);
                    am.y = __fadd_rn(am.y, o.dm.y);
                    am.z = __fadd_rn(am.z, o.dm.z);
                }
            }
        }
        dopac_out[i] = ado;
        if (dcov3D)
#pragma unroll
            for (int k = 0; k < 6; k++) dcov3D[6 * (size_t)i + k] = adc[k];
        if (want_sr) {
            dscale[3 * (size_t)i] = ads[0]; dscale[3 * (size_t)i + 1] = ads[1]; dscale[3 * (size_t)i + 2] = ads[2];
            drot[4 * (size_t)i] = adq.x; drot[4 * (size_t)i + 1] = adq.y;
            drot[4 * (size_t)i + 2] = adq.z; drot[4 * (size_t)i + 3] = adq.w;
        }
        if (!sh_follows) {
            dmean3D[3 * (size_t)i] = am.x; dmean3D[3 * (size_t)i + 1] = am.y; dmean3D[3 * (size_t)i + 2] = am.z;
        }
        if (dens.grad_sum && seen) {
            dens.grad_sum[i] = dg;
            dens.count[i] += seen;
            dens.flag[i] = 1;
        }
    }
}

// SH part (backward.cu:20-139 per view), two passes over the list that each hold
// one 48-float set (the coefficient sums or the SH row), not both.
// fold_shcoef_kernel: dL/dsh = the sum over views of basis x clamp-masked colour
// gradient (it depends only on the view direction).
__global__ void __launch_bounds__(128, 5)
    fold_shcoef_kernel(const FoldView* __restrict__ views, FoldView single, int nviews, int P,
                       const uint32_t* __restrict__ list, const unsigned long long* __restrict__ count,
                       const uint32_t* __restrict__ vis, float* __restrict__ dsh)
{
    const int words = (nviews + 31) >> 5;
    const PreParams& p = single.p;
    const int deg = p.D, M = p.M, nfl = M * 3;
    const int ncoef = (deg + 1) * (deg + 1);
    const bool vec = p.aligned && (nfl & 3) == 0;
    const uint32_t n = (uint32_t)*count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = (int)list[j];
        float acc[48];
#pragma unroll
        for (int f = 0; f < 48; f++) acc[f] = 0.f;
        const float3 mean = {p.means[3 * i], p.means[3 * i + 1], p.means[3 * i + 2]};
        for (int w = 0; w < words; w++) {
            uint32_t m = views_of(vis, w, P, i);
            while (m) {
                const int v = 32 * w + __ffs(m) - 1;
                m &= m - 1;
                const FoldView& fv = views ? views[v] : single;
                const float3 cam = {fv.p.campos[0], fv.p.campos[1], fv.p.campos[2]};
                float3 dir_orig;
                float x, y, z, B[16];
                sh_basis(mean, cam, dir_orig, x, y, z, B);
                const uint8_t cb = fv.clamped[i];
                const float d[3] = {(cb & 1) ? 0.f : fv.dcolor[3 * i], (cb & 2) ? 0.f : fv.dcolor[3 * i + 1],
                                    (cb & 4) ? 0.f : fv.dcolor[3 * i + 2]};
#pragma unroll
                for (int f = 0; f < 48; f++)
                    if (f < nfl) acc[f] = __fadd_rn(acc[f], sh_dsh(f, ncoef, B, d));
            }
        }
        float* drow = dsh + (size_t)i * nfl;
        if (vec) {
            float4* d4 = reinterpret_cast<float4*>(drow);
#pragma unroll
            for (int v = 0; v < 12; v++)
                if (4 * v < nfl) d4[v] = make_float4(acc[4 * v], acc[4 * v + 1], acc[4 * v + 2], acc[4 * v + 3]);
        } else {
#pragma unroll
            for (int f = 0; f < 48; f++)
                if (f < nfl) drow[f] = acc[f];
        }
    }
}

// fold_shdir_kernel: dL/dmean3D = the sum over views of (geometric term + the SH
// colour's dependence on the view direction); the SH row is read once.
__global__ void __launch_bounds__(128, 4)
    fold_shdir_kernel(const FoldView* __restrict__ views, FoldView single, int nviews, int P,
                      const uint32_t* __restrict__ list, const unsigned long long* __restrict__ count,
                      const uint32_t* __restrict__ vis, float* __restrict__ dmean3D)
{
    const int words = (nviews + 31) >> 5;
    const PreParams& p = single.p;
    const int deg = p.D, nfl = p.M * 3;
    const bool vec = p.aligned && (nfl & 3) == 0;
    const uint32_t n = (uint32_t)*count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = (int)list[j];
        float3 am = {0.f, 0.f, 0.f};
        float sh[48];
        if (deg > 0) load_sh_row(p.shs + (size_t)i * nfl, min(48, nfl), vec, sh);
        const float3 mean = {p.means[3 * i], p.means[3 * i + 1], p.means[3 * i + 2]};
        for (int w = 0; w < words; w++) {
            uint32_t m = views_of(vis, w, P, i);
            while (m) {
                const int v = 32 * w + __ffs(m) - 1;
                m &= m - 1;
                const FoldView& fv = views ? views[v] : single;
                float3 dmd = make_float3(0.f, 0.f, 0.f);
                if (deg > 0) {
                    const float3 cam = {fv.p.campos[0], fv.p.campos[1], fv.p.campos[2]};
                    float3 dir_orig;
                    float x, y, z;
                    sh_dir(mean, cam, dir_orig, x, y, z);
                    const uint8_t cb = fv.clamped[i];
                    const float d[3] = {(cb & 1) ? 0.f : fv.dcolor[3 * i], (cb & 2) ? 0.f : fv.dcolor[3 * i + 1],
                                        (cb & 4) ? 0.f : fv.dcolor[3 * i + 2]};
                    dmd = sh_ddir(deg, sh, x, y, z, d, dir_orig);
                }
                am.x = __fadd_rn(am.x, __fadd_rn(fv.dm_geo[3 * i], dmd.x));
                am.y = __fadd_rn(am.y, __fadd_rn(fv.dm_geo[3 * i + 1], dmd.y));
                am.z = __fadd_rn(am.z, __fadd_rn(fv.dm_geo[3 * i + 2], dmd.z));
            }
        }
        dmean3D[3 * (size_t)i] = am.x; dmean3D[3 * (size_t)i + 1] = am.y; dmean3D[3 * (size_t)i + 2] = am.z;
    }
}

// The Gaussians some view saw (any vis bit set), appended in any order to list
// (count[0] entries; the caller zeroes count).
__global__ void __launch_bounds__(256)
    seen_list_kernel(const uint32_t* __restrict__ vis, int words, int P, uint32_t* __restrict__ list,
                     unsigned long long* __restrict__ count)
{
    const int lane = threadIdx.x & 31;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < P; base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        bool any = false;
        if (i < P)
            for (int w = 0; w < words && !any; w++) any = vis[(size_t)w * P + i] != 0;
        const uint32_t b = __ballot_sync(0xffffffffu, any);
        if (!b) continue;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(count, (unsigned long long)__popc(b));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (any) list[at + __popc(b & ((1u << lane) - 1))] = (uint32_t)i;
    }
}

int grid_for(size_t n, int per_sm)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * per_sm));
}

// The two passes over the list (the caller has zeroed the output rows, which the
// passes overwrite for the listed Gaussians only).  list_bound sizes the grids.
void fold_launch(const FoldView* views, const FoldView& single, int nviews, int P, const uint32_t* list,
                 const unsigned long long* count, size_t list_bound, const uint32_t* vis, int consistent, bool sh,
                 float* dmean3D, float* dopac, float* dcov3D, float* dsh, float* dscale, float* drot,
                 const DensifyStats* dens, cudaStream_t s)
{
    // 128-thread blocks: these kernels hold 95-128 registers a thread
    const int blocks = 2 * grid_for(list_bound, 16);
    const DensifyStats d = dens ? *dens : DensifyStats{nullptr, nullptr, nullptr};
    fold_geo_kernel<<<blocks, 128, 0, s>>>(views, single, nviews, P, list, count, vis, consistent, sh, dmean3D, dopac,
                                           dcov3D, dscale, drot, d);
    if (sh) {
        fold_shcoef_kernel<<<blocks, 128, 0, s>>>(views, single, nviews, P, list, count, vis, dsh);
        fold_shdir_kernel<<<blocks, 128, 0, s>>>(views, single, nviews, P, list, count, vis, dmean3D);
    }
    note_launches(sh ? 3 : 1);
}

}  // namespace

void launch_preprocess_bwd(const PreParams& p, const GeomState& g, const float* pgrad, float* dmean2D,
                           float* dconic, float* dcolor, float* dopac, float* dmean3D, float* dcov3D, float* dsh,
                           float* dscale, float* drot, int consistent, cudaStream_t s)
{
    if (p.P <= 0) return;
    const bool sh = p.shs && dsh;
    pair_grad_gather_kernel<<<grid_for((size_t)p.P, 8), 256, 0, s>>>(g.sort_ids_b, g.total, g.pair_off, pgrad,
                                                                     dmean2D, dconic, dcolor, dopac, nullptr, 0u,
                                                                     0xffffffffu);
    note_launches(1);
    // the list: the view's visible Gaussians (depth order); the view's geometric
    // dL/dmean3D waits in the dL/dmean3D rows for the SH pass.  dL/dopacity is the
    // gather's output, read and rewritten in place (rows outside the list were
    // zeroed by the caller).
    const size_t P = (size_t)p.P;
    cudaMemsetAsync(dmean3D, 0, sizeof(float) * 3 * P, s);
    cudaMemsetAsync(dcov3D, 0, sizeof(float) * 6 * P, s);
    if (sh) cudaMemsetAsync(dsh, 0, sizeof(float) * 3 * (size_t)p.M * P, s);
    if (dscale) cudaMemsetAsync(dscale, 0, sizeof(float) * 3 * P, s);
    if (drot) cudaMemsetAsync(drot, 0, sizeof(float) * 4 * P, s);
    const FoldView one{p, dmean3D, dmean2D, dconic, dopac, dcolor, g.clamped};
    fold_launch(nullptr, one, 1, p.P, g.sort_ids_b, g.total + 1, P, nullptr, consistent, sh, dmean3D, dopac, dcov3D,
                dsh, dscale, drot, nullptr, s);
}

void launch_pair_grad_gather(const GeomState& g, const float* pgrad, long long rows, float* dmean2D, float* dconic,
                             float* dcolor, float* dopac, uint32_t* vis, uint32_t vis_bit, int P, cudaStream_t s)
{
    if (P <= 0) return;
    const uint32_t r = rows < 0 ? 0u : (rows > 0xffffffffll ? 0xffffffffu : (uint32_t)rows);
    pair_grad_gather_kernel<<<grid_for((size_t)P, 8), 256, 0, s>>>(g.sort_ids_b, g.total, g.pair_off, pgrad,
                                                                   dmean2D, dconic, dcolor, dopac, vis, vis_bit, r);
    note_launches(1);
}

void launch_fold_bwd(const FoldView* views, int nviews, int P, const uint32_t* vis, uint32_t* list,
                     unsigned long long* count, int consistent, bool sh, float* dmean3D, float* dopac, float* dsh,
                     float* dscale, float* drot, const DensifyStats* dens, const FoldView& shared, cudaStream_t s)
{
    if (P <= 0 || nviews <= 0) return;
    cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    seen_list_kernel<<<grid_for((size_t)P, 8), 256, 0, s>>>(vis, (nviews + 31) >> 5, P, list, count);
    note_launches(1);
    fold_launch(views, shared, nviews, P, list, count, (size_t)P, vis, consistent, sh, dmean3D, dopac, nullptr, dsh,
                dscale, drot, dens, s);
}

}  // namespace fgs
