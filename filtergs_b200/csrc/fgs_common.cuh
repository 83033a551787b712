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

// DILATE_PIXEL is a double literal in the reference: max() and += run in double.
__device__ __forceinline__ float dilate_max(float c) { return (float)fmax((double)c, 0.3); }
__device__ __forceinline__ float dilate_add(float c) { return (float)((double)c + 0.3); }

// Reduce 9 per-lane values over the warp with 16 shuffles instead of 45:
// a butterfly in which each level halves the values a lane keeps (the rest
// go to the partner lane).  Lanes 2s and 2s+1 end with the warp total of
// value s (s < 9; padded to 16 slots).
__device__ __forceinline__ float warp_transpose_sum9(const float (&g)[9])
{
    const unsigned lane = threadIdx.x & 31;
    float v[8];
    {
        const bool hi = lane & 16;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const float lo_v = g[i];
            const float hi_v = (i + 8 < 9) ? g[i + 8] : 0.f;
            const float send = hi ? lo_v : hi_v;
            const float keep = hi ? hi_v : lo_v;
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    }
#pragma unroll
    for (int w = 4, o = 8; w >= 1; w >>= 1, o >>= 1) {
        const bool hi = lane & o;
#pragma unroll
        for (int i = 0; i < w; i++) {
            const float send = hi ? v[i] : v[i + w];
            const float keep = hi ? v[i + w] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
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

// Colour of one Gaussian from its SH row `sh` ([M][3] floats).  Writes the
// per-channel clamp bits (bit c set when channel c was negative).
__device__ __forceinline__ float3 sh_to_rgb(int deg, const float* __restrict__ sh, float3 pos, float3 campos,
                                            uint8_t& clamp_bits)
{
    float3 dir = {pos.x - campos.x, pos.y - campos.y, pos.z - campos.z};
    const float len = sqrtf(dir.x * dir.x + dir.y * dir.y + dir.z * dir.z);
    dir.x = dir.x / len; dir.y = dir.y / len; dir.z = dir.z / len;
    float res[3];
#pragma unroll
    for (int c = 0; c < 3; c++) res[c] = kSH_C0 * sh[c];
    if (deg > 0) {
        const float x = dir.x, y = dir.y, z = dir.z;
#pragma unroll
        for (int c = 0; c < 3; c++)
            res[c] = res[c] - kSH_C1 * y * sh[3 + c] + kSH_C1 * z * sh[6 + c] - kSH_C1 * x * sh[9 + c];
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float xy = x * y, yz = y * z, xz = x * z;
#pragma unroll
            for (int c = 0; c < 3; c++)
                res[c] = res[c] + kSH_C2_0 * xy * sh[12 + c] + kSH_C2_1 * yz * sh[15 + c] +
                         kSH_C2_2 * (2.0f * zz - xx - yy) * sh[18 + c] + kSH_C2_3 * xz * sh[21 + c] +
                         kSH_C2_4 * (xx - yy) * sh[24 + c];
            if (deg > 2) {
#pragma unroll
                for (int c = 0; c < 3; c++)
                    res[c] = res[c] + kSH_C3_0 * y * (3.0f * xx - yy) * sh[27 + c] + kSH_C3_1 * xy * z * sh[30 + c] +
                             kSH_C3_2 * y * (4.0f * zz - xx - yy) * sh[33 + c] +
                             kSH_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * sh[36 + c] +
                             kSH_C3_4 * x * (4.0f * zz - xx - yy) * sh[39 + c] + kSH_C3_5 * z * (xx - yy) * sh[42 + c] +
                             kSH_C3_6 * x * (xx - 3.0f * yy) * sh[45 + c];
            }
        }
    }
    clamp_bits = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        res[c] += 0.5f;
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
