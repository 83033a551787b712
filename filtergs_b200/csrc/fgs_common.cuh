// Shared device helpers for the FilterGS rasterizer kernels (sm_100a).
//
// The projection / covariance arithmetic below is written in the same
// expression order as the reference (antialias/cuda_rasterizer/auxiliary.h,
// forward.cu, backward.cu and the glm 0.9.9 column-major mat3 product those
// use).  That order is what makes radii, tile rectangles and depth keys
// bit-identical with the reference build under the same nvcc FMA contraction,
// so it is kept even where a shorter form would do.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/filtergs_b200.h"

namespace fgs {

// Binning tile of the reference (config.h:16-17).  The OGFS radius formula
// always uses 256 (= 16*16) whatever tile the render kernels launch with.
constexpr int kTileX = 16;
constexpr int kTileY = 16;
constexpr int kOgfsBlockArea = 256;

// Bounded waits: every wait on another CTA or on a bulk copy gives up after
// kWaitLimitNs of the GPU's global timer and records FGS_ERR_TIMEOUT instead of
// hanging the GPU (legitimate waits last microseconds).
constexpr unsigned long long kWaitLimitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Deadline of one wait: expired() is called once per unsuccessful poll and
// reads the timer every 256 polls (the first read starts the clock).
struct WaitBound {
    unsigned long long t0 = 0;
    uint32_t polls = 0;
    __device__ __forceinline__ bool expired(unsigned long long limit_ns)
    {
        if ((++polls & 255u) != 0) return false;
        const unsigned long long t = global_ns();
        if (t0 == 0) {
            t0 = t;
            return false;
        }
        return t - t0 > limit_ns;
    }
};

__device__ __forceinline__ void set_error(unsigned int* err, unsigned int code)
{
    if (err) atomicOr(err, 1u << code);
}

// ---------------------------------------------------------------- pinned multiply-add grouping
// The reference build leaves the fusion of its sums of products to nvcc.  Where
// an output must equal the reference's bits, the grouping nvcc chose there (found
// by comparing candidate groupings with the reference build's outputs) is written
// out with round-to-nearest intrinsics, which the compiler never re-fuses.
//   dot3<M>:  ((a0 b0 + a1 b1) + a2 b2); M / 2 picks the inner step (0: a0 b0 fused
//             into the add, 1: a1 b1 fused, 2: no fusion), M % 2 the outer one
//             (0: a2 b2 fused, 1: not).
//   sum2<M>:  a b + c d; M = 0: a b fused, 1: c d fused, 2: no fusion.
template <int M>
__device__ __forceinline__ float dot3(float a0, float b0, float a1, float b1, float a2, float b2)
{
    float x;
    if constexpr (M / 2 == 0) x = __fmaf_rn(a0, b0, __fmul_rn(a1, b1));
    else if constexpr (M / 2 == 1) x = __fmaf_rn(a1, b1, __fmul_rn(a0, b0));
    else x = __fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1));
    if constexpr (M % 2 == 0) return __fmaf_rn(a2, b2, x);
    else return __fadd_rn(x, __fmul_rn(a2, b2));
}
template <int M>
__device__ __forceinline__ float sum2(float a, float b, float c, float d)
{
    if constexpr (M == 0) return __fmaf_rn(a, b, __fmul_rn(c, d));
    else if constexpr (M == 1) return __fmaf_rn(c, d, __fmul_rn(a, b));
    else return __fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d));
}

// ---------------------------------------------------------------- 4x4 transforms
// Column-major 16-float matrices as stored by the reference (auxiliary.h:58-106).
__device__ __forceinline__ float3 xform_point4x3(const float3& p, const float* m)
{
    return {m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
            m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
            m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]};
}
__device__ __forceinline__ float4 xform_point4x4(const float3& p, const float* m)
{
    return {m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
            m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
            m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14],
            m[3] * p.x + m[7] * p.y + m[11] * p.z + m[15]};
}

// auxiliary.h:41-44: the double literals make this a double-precision expression.
__device__ __forceinline__ float ndc_to_pix(float v, int S)
{
    return ((v + 1.0) * S - 1.0) * 0.5;
}

// auxiliary.h:46-56 with the tile extent as a parameter (float division by
// the tile size, then truncation toward zero, then clamping to the grid).
__device__ __forceinline__ void tile_rect(float px, float py, int r, int gx, int gy, int tx, int ty,
                                          int& x0, int& y0, int& x1, int& y1)
{
    x0 = min(gx, max(0, (int)((px - r) / tx)));
    y0 = min(gy, max(0, (int)((py - r) / ty)));
    x1 = min(gx, max(0, (int)((px + r + tx - 1) / tx)));
    y1 = min(gy, max(0, (int)((py + r + ty - 1) / ty)));
}

// ---------------------------------------------------------------- 3x3 (glm order)
// m[c][r]: column c, row r.  mul() is glm's mat3*mat3 term by term.
struct M3 {
    float m[3][3];
};
__device__ __forceinline__ M3 m3_cols(float a0, float a1, float a2, float b0, float b1, float b2, float c0,
                                      float c1, float c2)
{
    M3 r;
    r.m[0][0] = a0; r.m[0][1] = a1; r.m[0][2] = a2;
    r.m[1][0] = b0; r.m[1][1] = b1; r.m[1][2] = b2;
    r.m[2][0] = c0; r.m[2][1] = c1; r.m[2][2] = c2;
    return r;
}
__device__ __forceinline__ M3 m3_mul(const M3& A, const M3& B)
{
    M3 R;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++)
            R.m[c][r] = A.m[0][r] * B.m[c][0] + A.m[1][r] * B.m[c][1] + A.m[2][r] * B.m[c][2];
    return R;
}
__device__ __forceinline__ M3 m3_t(const M3& A)
{
    M3 R;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) R.m[c][r] = A.m[r][c];
    return R;
}

// forward.cu:151-185 -- quaternion (r,x,y,z) used as given.
__device__ __forceinline__ void cov3d_from_scale_rot(float sx, float sy, float sz, float mod, float4 q,
                                                     float cov[6])
{
    M3 S = m3_cols(1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f);
    S.m[0][0] = mod * sx;
    S.m[1][1] = mod * sy;
    S.m[2][2] = mod * sz;
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    M3 R = m3_cols(1.f - 2.f * (y * y + z * z), 2.f * (x * y - r * z), 2.f * (x * z + r * y),
                   2.f * (x * y + r * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - r * x),
                   2.f * (x * z - r * y), 2.f * (y * z + r * x), 1.f - 2.f * (x * x + y * y));
    M3 M = m3_mul(S, R);
    M3 Sig = m3_mul(m3_t(M), M);
    cov[0] = Sig.m[0][0]; cov[1] = Sig.m[0][1]; cov[2] = Sig.m[0][2];
    cov[3] = Sig.m[1][1]; cov[4] = Sig.m[1][2]; cov[5] = Sig.m[2][2];
}

// EWA projection (forward.cu:102-146).  Returns the un-dilated cov2D entries
// (c00, c01, c11) and, optionally, T = W*J and the clamp state for backward.
struct Ewa {
    M3 T;
    float tx, ty, tz;
    float txtz, tytz;
    bool xclamp, yclamp;
};
__device__ __forceinline__ float3 ewa_cov2d(const float3& mean, float fx, float fy, float tanx, float tany,
                                            const float* cov3D, const float* view, Ewa* e = nullptr)
{
    float3 t = xform_point4x3(mean, view);
    const float limx = 1.3f * tanx;
    const float limy = 1.3f * tany;
    const float txtz = t.x / t.z;
    const float tytz = t.y / t.z;
    t.x = fminf(limx, fmaxf(-limx, txtz)) * t.z;
    t.y = fminf(limy, fmaxf(-limy, tytz)) * t.z;
    M3 J = m3_cols(fx / t.z, 0.0f, -(fx * t.x) / (t.z * t.z), 0.0f, fy / t.z, -(fy * t.y) / (t.z * t.z), 0, 0, 0);
    M3 W = m3_cols(view[0], view[4], view[8], view[1], view[5], view[9], view[2], view[6], view[10]);
    M3 T = m3_mul(W, J);
    M3 V = m3_cols(cov3D[0], cov3D[1], cov3D[2], cov3D[1], cov3D[3], cov3D[4], cov3D[2], cov3D[4], cov3D[5]);
    M3 C = m3_mul(m3_mul(m3_t(T), m3_t(V)), T);
    if (e) {
        e->T = T;
        e->tx = t.x; e->ty = t.y; e->tz = t.z;
        e->txtz = txtz; e->tytz = tytz;
        e->xclamp = txtz < -limx || txtz > limx;
        e->yclamp = tytz < -limy || tytz > limy;
    }
    return {C.m[0][0], C.m[0][1], C.m[1][1]};
}

// The forward preprocess's covariance chain with the reference build's grouping
// spelled out (found by comparing candidate groupings with the reference build's
// cov3D and conic outputs; every visible Gaussian of three 1080p views of the
// 2M-Gaussian scene agrees bit for bit).  cov3d_ref: computeCov3D (forward.cu:151-185):
// in the rotation matrix the products shared by two entries (y y, z z; x z) are the
// ones left unfused, M = S R takes one product per entry, Sigma = M^T M fuses the
// first and last products of each dot.  ewa_cov2d_ref: computeCov2D
// (forward.cu:102-146) with every dot fusing its first and last product.
__device__ __forceinline__ void cov3d_ref(float sx, float sy, float sz, float mod, float4 q, float cov[6])
{
    const float r = q.x, x = q.y, y = q.z, z = q.w;
    float R[3][3];  // R[c][k]: glm column c, row k
    R[0][0] = __fsub_rn(1.f, __fmul_rn(2.f, sum2<2>(y, y, z, z)));
    R[0][1] = __fmul_rn(2.f, sum2<0>(x, y, -r, z));
    R[0][2] = __fmul_rn(2.f, sum2<1>(x, z, r, y));
    R[1][0] = __fmul_rn(2.f, sum2<0>(x, y, r, z));
    R[1][1] = __fsub_rn(1.f, __fmul_rn(2.f, sum2<0>(x, x, z, z)));
    R[1][2] = __fmul_rn(2.f, sum2<0>(y, z, -r, x));
    R[2][0] = __fmul_rn(2.f, sum2<1>(x, z, -r, y));
    R[2][1] = __fmul_rn(2.f, sum2<0>(y, z, r, x));
    R[2][2] = __fsub_rn(1.f, __fmul_rn(2.f, sum2<0>(x, x, y, y)));
    const float s[3] = {__fmul_rn(mod, sx), __fmul_rn(mod, sy), __fmul_rn(mod, sz)};
    float M[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int k = 0; k < 3; k++) M[c][k] = __fmul_rn(s[k], R[c][k]);
    auto sig = [&](int c, int k) { return dot3<0>(M[k][0], M[c][0], M[k][1], M[c][1], M[k][2], M[c][2]); };
    cov[0] = sig(0, 0); cov[1] = sig(0, 1); cov[2] = sig(0, 2);
    cov[3] = sig(1, 1); cov[4] = sig(1, 2); cov[5] = sig(2, 2);
}

__device__ __forceinline__ float3 ewa_cov2d_ref(const float3& mean, float fx, float fy, float tanx, float tany,
                                                const float* cov3D, const float* v)
{
    float tx = __fadd_rn(dot3<0>(v[0], mean.x, v[4], mean.y, v[8], mean.z), v[12]);
    float ty = __fadd_rn(dot3<0>(v[1], mean.x, v[5], mean.y, v[9], mean.z), v[13]);
    const float tz = __fadd_rn(dot3<0>(v[2], mean.x, v[6], mean.y, v[10], mean.z), v[14]);
    const float limx = __fmul_rn(1.3f, tanx), limy = __fmul_rn(1.3f, tany);
    tx = __fmul_rn(fminf(limx, fmaxf(-limx, __fdiv_rn(tx, tz))), tz);
    ty = __fmul_rn(fminf(limy, fmaxf(-limy, __fdiv_rn(ty, tz))), tz);
    const float tz2 = __fmul_rn(tz, tz);
    const float j00 = __fdiv_rn(fx, tz), j02 = __fdiv_rn(-__fmul_rn(fx, tx), tz2);
    const float j11 = __fdiv_rn(fy, tz), j12 = __fdiv_rn(-__fmul_rn(fy, ty), tz2);
    // T = W J (W[c][k] = v[4k + c]); J's zero entries add exact zeros
    float T[2][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T[0][k] = __fmaf_rn(v[4 * k + 2], j02, __fmul_rn(v[4 * k], j00));
        T[1][k] = __fmaf_rn(v[4 * k + 2], j12, __fmul_rn(v[4 * k + 1], j11));
    }
    const float V[3][3] = {{cov3D[0], cov3D[1], cov3D[2]}, {cov3D[1], cov3D[3], cov3D[4]},
                           {cov3D[2], cov3D[4], cov3D[5]}};
    float X[3][2];  // X = T^T V^T (rows 0, 1)
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int k = 0; k < 2; k++) X[c][k] = dot3<0>(T[k][0], V[0][c], T[k][1], V[1][c], T[k][2], V[2][c]);
    auto cv = [&](int c, int k) { return dot3<0>(X[0][k], T[c][0], X[1][k], T[c][1], X[2][k], T[c][2]); };
    return {cv(0, 0), cv(0, 1), cv(1, 1)};
}

// DILATE_PIXEL is a double literal in the reference: max() and += run in double.
__device__ __forceinline__ float dilate_max(float c) { return (float)fmax((double)c, 0.3); }
__device__ __forceinline__ float dilate_add(float c) { return (float)((double)c + 0.3); }

// One level of warp_transpose_sum9: lanes with bit `o` clear keep values
// [0, M) of the N they hold, the others keep [M, N) (padded with zeros to M),
// each adding the partner lane's copy of what it keeps.
template <int M, int N>
__device__ __forceinline__ void sum9_level(const float (&in)[N], float (&out)[M], unsigned lane, int o)
{
    const bool hi = lane & o;
#pragma unroll
    for (int i = 0; i < M; i++) {
        const float lo_v = in[i];
        const float hi_v = i + M < N ? in[i + M] : 0.f;
        const float send = hi ? lo_v : hi_v;
        const float keep = hi ? hi_v : lo_v;
        out[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
}

// Reduce 9 per-lane values over the warp with 12 shuffles instead of 45: a
// butterfly in which each level splits the values a lane holds as evenly as
// it can (9 -> 5/4 -> 3/2 -> 2/1 -> 1) and sends the other part to the partner
// lane, then one plain butterfly step.  Lanes 2s and 2s+1 end with the warp
// total of value sum9_component(2s) (values past 8 are padding).
__device__ __forceinline__ float warp_transpose_sum9(const float (&g)[9])
{
    const unsigned lane = threadIdx.x & 31;
    float v5[5], v3[3], v2[2], v1[1];
    sum9_level<5, 9>(g, v5, lane, 16);
    sum9_level<3, 5>(v5, v3, lane, 8);
    sum9_level<2, 3>(v3, v2, lane, 4);
    sum9_level<1, 2>(v2, v1, lane, 2);
    return v1[0] + __shfl_xor_sync(0xffffffffu, v1[0], 1);
}

// Which of the nine values warp_transpose_sum9 leaves on `lane` (15: padding).
// Lane bits 4, 3, 2, 1 pick offsets 5, 3, 2, 1 inside the split at that level.
__device__ __forceinline__ int sum9_component(unsigned lane)
{
    return (int)((0xfff8f765ff43f210ull >> (4 * ((lane & 31) >> 1))) & 15u);
}

// ---------------------------------------------------------------- SH (forward.cu:48-99)
__device__ constexpr float kSH_C0 = 0.28209479177387814f;
__device__ constexpr float kSH_C1 = 0.4886025119029199f;
__device__ constexpr float kSH_C2_0 = 1.0925484305920792f;
__device__ constexpr float kSH_C2_1 = -1.0925484305920792f;
__device__ constexpr float kSH_C2_2 = 0.31539156525252005f;
__device__ constexpr float kSH_C2_3 = -1.0925484305920792f;
__device__ constexpr float kSH_C2_4 = 0.5462742152960396f;
__device__ constexpr float kSH_C3_0 = -0.5900435899266435f;
__device__ constexpr float kSH_C3_1 = 2.890611442640554f;
__device__ constexpr float kSH_C3_2 = -0.4570457994644658f;
__device__ constexpr float kSH_C3_3 = 0.3731763325901154f;
__device__ constexpr float kSH_C3_4 = -0.4570457994644658f;
__device__ constexpr float kSH_C3_5 = 1.445305721320277f;
__device__ constexpr float kSH_C3_6 = -0.5900435899266435f;

// Colour of one Gaussian from its SH row `sh` ([M][3] floats) -- computeColorFromSH
// (forward.cu:48-99) with the multiply-add grouping of the reference build spelled
// out (found by comparing candidate groupings with the reference build's colours:
// every visible Gaussian of three 1080p views of the 2M-Gaussian scene agrees bit
// for bit).  Writes the per-channel clamp bits (bit c set when channel c was
// negative).
__device__ __forceinline__ float3 sh_to_rgb(int deg, const float* __restrict__ sh, float3 pos, float3 campos,
                                            uint8_t& clamp_bits)
{
    float3 dir = {__fsub_rn(pos.x, campos.x), __fsub_rn(pos.y, campos.y), __fsub_rn(pos.z, campos.z)};
    const float len = __fsqrt_rn(dot3<0>(dir.x, dir.x, dir.y, dir.y, dir.z, dir.z));  // glm::length
    dir.x = __fdiv_rn(dir.x, len); dir.y = __fdiv_rn(dir.y, len); dir.z = __fdiv_rn(dir.z, len);
    float res[3];
#pragma unroll
    for (int c = 0; c < 3; c++) res[c] = __fmul_rn(kSH_C0, sh[c]);
    if (deg > 0) {
        const float x = dir.x, y = dir.y, z = dir.z;
        const float c1y = __fmul_rn(kSH_C1, y), c1z = __fmul_rn(kSH_C1, z), c1x = __fmul_rn(kSH_C1, x);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            // result - C1 y sh1 + C1 z sh2 - C1 x sh3: the first product of the chain is the one fused
            float r = __fmaf_rn(-c1y, sh[3 + c], res[c]);
            r = __fmaf_rn(c1z, sh[6 + c], r);
            res[c] = __fmaf_rn(-c1x, sh[9 + c], r);
        }
        if (deg > 1) {
            const float xx = __fmul_rn(x, x), yy = __fmul_rn(y, y), zz = __fmul_rn(z, z);
            const float xy = __fmul_rn(x, y), yz = __fmul_rn(y, z), xz = __fmul_rn(x, z);
            const float f0 = __fmul_rn(kSH_C2_0, xy), f1 = __fmul_rn(kSH_C2_1, yz);
            const float f2 = __fmul_rn(kSH_C2_2, __fsub_rn(__fsub_rn(__fmul_rn(2.0f, zz), xx), yy));
            const float f3 = __fmul_rn(kSH_C2_3, xz), f4 = __fmul_rn(kSH_C2_4, __fsub_rn(xx, yy));
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float r = __fmaf_rn(f0, sh[12 + c], res[c]);
                r = __fmaf_rn(f1, sh[15 + c], r);
                r = __fmaf_rn(f2, sh[18 + c], r);
                r = __fmaf_rn(f3, sh[21 + c], r);
                res[c] = __fmaf_rn(f4, sh[24 + c], r);
            }
            if (deg > 2) {
                const float q4 = __fsub_rn(__fsub_rn(__fmul_rn(4.0f, zz), xx), yy);  // 4 zz - xx - yy
                const float g0 = __fmul_rn(__fmul_rn(kSH_C3_0, y), __fmaf_rn(3.0f, xx, -yy));
                const float g1 = __fmul_rn(__fmul_rn(kSH_C3_1, xy), z);
                const float g2 = __fmul_rn(__fmul_rn(kSH_C3_2, y), q4);
                const float g3 = __fmul_rn(__fmul_rn(kSH_C3_3, z),
                                           __fmaf_rn(-3.0f, yy, __fmaf_rn(-3.0f, xx, __fmul_rn(2.0f, zz))));
                const float g4 = __fmul_rn(__fmul_rn(kSH_C3_4, x), q4);
                const float g5 = __fmul_rn(__fmul_rn(kSH_C3_5, z), __fsub_rn(xx, yy));
                const float g6 = __fmul_rn(__fmul_rn(kSH_C3_6, x), __fmaf_rn(-3.0f, yy, xx));
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float r = __fmaf_rn(g0, sh[27 + c], res[c]);
                    r = __fmaf_rn(g1, sh[30 + c], r);
                    r = __fmaf_rn(g2, sh[33 + c], r);
                    r = __fmaf_rn(g3, sh[36 + c], r);
                    r = __fmaf_rn(g4, sh[39 + c], r);
                    r = __fmaf_rn(g5, sh[42 + c], r);
                    res[c] = __fmaf_rn(g6, sh[45 + c], r);
                }
            }
        }
    }
    clamp_bits = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        res[c] = __fadd_rn(res[c], 0.5f);
        if (res[c] < 0) clamp_bits |= (uint8_t)(1u << c);
    }
    return {fmaxf(res[0], 0.0f), fmaxf(res[1], 0.0f), fmaxf(res[2], 0.0f)};
}

// ---------------------------------------------------------------- render records
// One sorted (tile, Gaussian) pair as the render kernels stage it: 48 bytes,
// 16-byte aligned so a batch is one contiguous bulk copy.
struct __align__(16) PairRecord {
    float4 a;  // x, y, conic.x, conic.y
    float4 b;  // conic.z, opacity, r, g
    float4 c;  // b, gaussian id (bits), 0, 0
};
static_assert(sizeof(PairRecord) == 48, "record size");

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }

}  // namespace fgs
