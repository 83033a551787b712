// Training-step kernels around the rasterizer (the loss, the optimizer and the
// densification statistics of LoG's training loop):
//
//   loss       LoG/render/loss.py:6-44 (SSIM, 11x11 Gaussian window, sigma 1.5,
//              no padding: "valid" outputs) and renderer.py:260-273
//              (0.8 * L1 + 0.2 * (1 - SSIM)), forward and gradient in two tiled
//              kernels per image channel, partial sums reduced in a fixed order.
//   activate   LoG/model/activation.py (exp scale, sigmoid opacity, normalised
//              quaternion) from the raw parameters.
//   adam       LoG/model/sparse_optimizer.py:41-78,163-196: Adam with bias
//              correction from the global step, eps 1e-15, on the rows that were
//              visible this step only; the gradients w.r.t. the activated values
//              are chained through the activations first, and the activated values
//              of the updated rows are rewritten for the next forward.
//   densify    LoG/model/counter.py:36-83 (reduced to the two statistics the
//              training step keeps): sum of |dL/dmean2D[:, :2]| and the visibility
//              count per Gaussian, plus this step's visible flag.
#include <cmath>

#include "fgs_common.cuh"
#include "fgs_internal.h"

namespace fgs {

namespace {

constexpr int kWin = 11;           // SSIM window
constexpr int kHalo = kWin - 1;    // valid outputs lose kHalo rows / columns
constexpr int kTX = 32, kTY = 16;  // output (or pixel) tile of one CTA
constexpr float kC1 = 0.01f * 0.01f, kC2 = 0.03f * 0.03f;

struct Window {
    float g[kWin];
};

// ---------------------------------------------------------------- SSIM forward + coefficient maps
// One CTA: a kTX x kTY tile of valid outputs of one channel, kTX x kTY / kRowsPer
// threads.  The input tile with its halo is staged in shared memory, the 11-tap
// Gaussian is applied along rows, then along columns (separable) to x, y, x^2, y^2
// and x*y, each pass from a sliding window in registers (a row item makes kSeg
// outputs from kSeg + 10 loaded values, a thread kRowsPer outputs of one column from
// kRowsPer + 10), every output summing its taps in window order.  Per output q the
// loss gradient w.r.t. the five local means is kept as three maps (d/dmu_x,
// d/dE[x^2], d/dE[xy]); the SSIM values of the tile are summed in a fixed order.
constexpr int kRowsPer = 4;                       // outputs of one column per thread
constexpr int kLossThreads = kTX * kTY / kRowsPer;
constexpr int kSeg = 8;                           // outputs of one row per row-pass item

__global__ void __launch_bounds__(kLossThreads)
    ssim_forward_kernel(int W, int H, const float* __restrict__ pred, const float* __restrict__ target, Window win,
                        float ssim_grad_scale, float* __restrict__ gmap, float* __restrict__ partial)
{
    __shared__ float sx[kTY + kHalo][kTX + kHalo + 1];
    __shared__ float sy[kTY + kHalo][kTX + kHalo + 1];
    __shared__ float hq[5][kTY + kHalo][kTX];
    __shared__ float red[kLossThreads / 32];
    const int Wo = W - kHalo, Ho = H - kHalo;
    const int c = blockIdx.z;
    const int ox0 = blockIdx.x * kTX, oy0 = blockIdx.y * kTY;
    const float* x = pred + (size_t)c * W * H;
    const float* y = target + (size_t)c * W * H;
    const int tid = threadIdx.x;
    for (int i = tid; i < (kTY + kHalo) * (kTX + kHalo); i += kLossThreads) {
        const int r = i / (kTX + kHalo), cc = i % (kTX + kHalo);
        const int gy = oy0 + r, gx = ox0 + cc;
        const bool in = gy < H && gx < W;
        sx[r][cc] = in ? __ldg(x + (size_t)gy * W + gx) : 0.f;
        sy[r][cc] = in ? __ldg(y + (size_t)gy * W + gx) : 0.f;
    }
    __syncthreads();
    for (int i = tid; i < (kTY + kHalo) * (kTX / kSeg); i += kLossThreads) {
        const int r = i / (kTX / kSeg), c0 = (i % (kTX / kSeg)) * kSeg;
        float u[kSeg + kHalo], v[kSeg + kHalo];
#pragma unroll
        for (int k = 0; k < kSeg + kHalo; k++) {
            u[k] = sx[r][c0 + k];
            v[k] = sy[r][c0 + k];
        }
#pragma unroll
        for (int k = 0; k < kSeg; k++) {
            float a = 0.f, b = 0.f, aa = 0.f, bb = 0.f, ab = 0.f;
#pragma unroll
            for (int j = 0; j < kWin; j++) {
                const float uu = u[k + j], vv = v[k + j], w = win.g[j];
                a += w * uu;
                b += w * vv;
                aa += w * (uu * uu);
                bb += w * (vv * vv);
                ab += w * (uu * vv);
            }
            hq[0][r][c0 + k] = a; hq[1][r][c0 + k] = b; hq[2][r][c0 + k] = aa; hq[3][r][c0 + k] = bb;
            hq[4][r][c0 + k] = ab;
        }
    }
    __syncthreads();
    const int tx = tid % kTX, ty0 = (tid / kTX) * kRowsPer;
    float m[kRowsPer][5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        float col[kRowsPer + kHalo];
#pragma unroll
        for (int k = 0; k < kRowsPer + kHalo; k++) col[k] = hq[q][ty0 + k][tx];
#pragma unroll
        for (int rr = 0; rr < kRowsPer; rr++) {
            float acc = 0.f;
#pragma unroll
            for (int i = 0; i < kWin; i++) acc += win.g[i] * col[rr + i];
            m[rr][q] = acc;
        }
    }
    float s = 0.f;
    const size_t plane = (size_t)Wo * Ho;
    float* gm = gmap + (size_t)c * 3 * plane;
#pragma unroll
    for (int rr = 0; rr < kRowsPer; rr++) {
        const int ox = ox0 + tx, oy = oy0 + ty0 + rr;
        if (ox < Wo && oy < Ho) {
            const float m1 = m[rr][0], m2 = m[rr][1];
            const float s11 = m[rr][2] - m1 * m1, s22 = m[rr][3] - m2 * m2, s12 = m[rr][4] - m1 * m2;
            const float A = 2.f * m1 * m2 + kC1, B = 2.f * s12 + kC2;
            const float Cc = m1 * m1 + m2 * m2 + kC1, D = s11 + s22 + kC2;
            const float CD = Cc * D;
            const float ss = (A * B) / CD;
            // d ssim / d(mu_x, E[x^2], E[xy]); the loss is 0.2 (1 - mean ssim): scale by -ssim_grad_scale
            const float d_m1 = (2.f * m2 * B - 2.f * m2 * A) / CD - ss * (2.f * m1 / Cc - 2.f * m1 / D);
            const float d_e11 = -ss / D;
            const float d_e12 = 2.f * A / CD;
            const size_t o = (size_t)oy * Wo + ox;
            gm[o] = -ssim_grad_scale * d_m1;
            gm[plane + o] = -ssim_grad_scale * d_e11;
            gm[2 * plane + o] = -ssim_grad_scale * d_e12;
            s += ss;
        }
    }
    // fixed-order block sum of the tile's SSIM values
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        float t = 0.f;
        for (int w = 0; w < kLossThreads / 32; w++) t += red[w];
        partial[((size_t)c * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
    }
}

// ---------------------------------------------------------------- loss gradient per pixel
// dL/dx_p = sum over the outputs q whose window covers p of w(q, p) *
// (G1(q) + 2 x_p G11(q) + y_p G12(q)), a transposed separable convolution of the
// three coefficient maps, plus the L1 term w_l1 * sign(x_p - y_p).  One CTA: a
// kTX x kTY pixel tile of one channel, the two passes from sliding windows in
// registers as in ssim_forward_kernel; also sums |x - y| over the tile.
__global__ void __launch_bounds__(kLossThreads)
    loss_grad_kernel(int W, int H, const float* __restrict__ pred, const float* __restrict__ target, Window win,
                     const float* __restrict__ gmap, float l1_grad_scale, float* __restrict__ dpred,
                     float* __restrict__ partial)
{
    __shared__ float sg[3][kTY + kHalo][kTX + kHalo + 1];
    __shared__ float hv[3][kTY + kHalo][kTX];
    __shared__ float red[kLossThreads / 32];
    const int Wo = W - kHalo, Ho = H - kHalo;
    const int c = blockIdx.z;
    const int px0 = blockIdx.x * kTX, py0 = blockIdx.y * kTY;
    const size_t plane = (size_t)Wo * Ho;
    const float* gm = gmap + (size_t)c * 3 * plane;
    const int tid = threadIdx.x;
    // outputs q in [p - kHalo, p]: rows py0 - kHalo .. py0 + kTY - 1
    for (int i = tid; i < (kTY + kHalo) * (kTX + kHalo); i += kLossThreads) {
        const int r = i / (kTX + kHalo), cc = i % (kTX + kHalo);
        const int qy = py0 - kHalo + r, qx = px0 - kHalo + cc;
        const bool in = qy >= 0 && qx >= 0 && qy < Ho && qx < Wo;
        const size_t o = (size_t)qy * Wo + qx;
#pragma unroll
        for (int k = 0; k < 3; k++) sg[k][r][cc] = in ? __ldg(gm + k * plane + o) : 0.f;
    }
    __syncthreads();
    // along rows: T(r, p) = sum_j g_j G(r, p - j), window sg[r][c0 .. c0 + kSeg + kHalo)
    for (int i = tid; i < (kTY + kHalo) * (kTX / kSeg); i += kLossThreads) {
        const int r = i / (kTX / kSeg), c0 = (i % (kTX / kSeg)) * kSeg;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float g[kSeg + kHalo];
#pragma unroll
            for (int e = 0; e < kSeg + kHalo; e++) g[e] = sg[k][r][c0 + e];
#pragma unroll
            for (int kk = 0; kk < kSeg; kk++) {
                float t = 0.f;
#pragma unroll
                for (int jj = 0; jj < kWin; jj++) t += win.g[jj] * g[kk + kHalo - jj];
                hv[k][r][c0 + kk] = t;
            }
        }
    }
    __syncthreads();
    const int tx = tid % kTX, ty0 = (tid / kTX) * kRowsPer;
    float sv[kRowsPer][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float col[kRowsPer + kHalo];
#pragma unroll
        for (int e = 0; e < kRowsPer + kHalo; e++) col[e] = hv[k][ty0 + e][tx];
#pragma unroll
        for (int rr = 0; rr < kRowsPer; rr++) {
            float acc = 0.f;
#pragma unroll
            for (int ii = 0; ii < kWin; ii++) acc += win.g[ii] * col[rr + kHalo - ii];
            sv[rr][k] = acc;
        }
    }
    float l1 = 0.f;
#pragma unroll
    for (int rr = 0; rr < kRowsPer; rr++) {
        const int px = px0 + tx, py = py0 + ty0 + rr;
        if (px < W && py < H) {
            const size_t o = (size_t)c * W * H + (size_t)py * W + px;
            const float xv = __ldg(pred + o), yv = __ldg(target + o);
            const float d = xv - yv;
            const float sgn = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
            dpred[o] = sv[rr][0] + 2.f * xv * sv[rr][1] + yv * sv[rr][2] + l1_grad_scale * sgn;
            l1 += fabsf(d);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l1 += __shfl_xor_sync(0xffffffffu, l1, o);
    if ((tid & 31) == 0) red[tid >> 5] = l1;
    __syncthreads();
    if (tid == 0) {
        float t = 0.f;
        for (int w = 0; w < kLossThreads / 32; w++) t += red[w];
        partial[((size_t)c * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
    }
}

// sums[0] += sum(l1 partials), sums[1] += sum(ssim partials), by one block in a
// fixed order: thread t adds partials t, t + blockDim.x, ... in turn, a butterfly of
// shuffles adds the warp's 32 values (every lane ends with the same bits: each step
// adds the same two operands on both lanes), and thread 0 adds the warp totals in
// warp order.  Every call with the same partials gives the same sums.
__global__ void __launch_bounds__(1024) loss_reduce_kernel(const float* __restrict__ l1p, int nl1,
                                                           const float* __restrict__ sp, int ns,
                                                           double* __restrict__ sums)
{
    __shared__ double s_a[32], s_b[32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nl1; i += blockDim.x) a += l1p[i];
    for (int i = threadIdx.x; i < ns; i += blockDim.x) b += sp[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_a[threadIdx.x >> 5] = a;
        s_b[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            ta += s_a[w];
            tb += s_b[w];
        }
        sums[0] += ta;
        sums[1] += tb;
    }
}

// ---------------------------------------------------------------- activation, densification, Adam
__device__ __forceinline__ float sigmoidf(float x) { return 1.f / (1.f + expf(-x)); }

__global__ void activate_kernel(int P, const float* __restrict__ log_scale, const float* __restrict__ rot_raw,
                                const float* __restrict__ opac_logit, float* __restrict__ scale,
                                float* __restrict__ rot, float* __restrict__ opac)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; k++) scale[3 * i + k] = expf(log_scale[3 * i + k]);
        const float q0 = rot_raw[4 * i], q1 = rot_raw[4 * i + 1], q2 = rot_raw[4 * i + 2], q3 = rot_raw[4 * i + 3];
        const float n = fmaxf(sqrtf(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3), 1e-12f);
        rot[4 * i] = q0 / n; rot[4 * i + 1] = q1 / n; rot[4 * i + 2] = q2 / n; rot[4 * i + 3] = q3 / n;
        opac[i] = sigmoidf(opac_logit[i]);
    }
}

// Plain path: one view's dense screen-space gradient and radii.
__global__ void densify_dense_kernel(int P, const int* __restrict__ radii, const float* __restrict__ dmean2D,
                                     float* __restrict__ grad_sum, int* __restrict__ vis_count,
                                     uint8_t* __restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        if (radii[i] <= 0) continue;
        const float gx = dmean2D[3 * i], gy = dmean2D[3 * i + 1];
        grad_sum[i] += sqrtf(gx * gx + gy * gy);
        vis_count[i] += 1;
        flag[i] = 1;
    }
}

struct AdamRow {
    float* p;
    float* m;
    float* v;
};

// sparse_optimizer.py:54-76 with torch's float32 arithmetic: the Python-float
// coefficients beta and 1 - beta (formed in double) are rounded to float.
__device__ __forceinline__ void adam_update(float& p, float& m, float& v, float g, float b1, float omb1, float b2,
                                            float omb2, float step_size, float bc2_sqrt, float eps)
{
    m = m * b1 + g * omb1;
    v = v * b2 + omb2 * g * g;
    const float denom = sqrtf(v) / bc2_sqrt + eps;
    p = p + (-step_size) * (m / denom);
}

}  // namespace

// Bias corrections of the global step, as the reference forms them (double), and the
// float coefficients of the update.
struct AdamCoef {
    double bc1;
    float bc2s, b1, b2, omb1, omb2, eps;
};

__device__ __forceinline__ AdamCoef adam_coef(const fgs_adam_args& a, int t)
{
    AdamCoef c;
    c.bc1 = 1.0 - pow(a.beta1, (double)t);
    c.bc2s = (float)sqrt(1.0 - pow(a.beta2, (double)t));
    c.b1 = (float)a.beta1;
    c.b2 = (float)a.beta2;
    c.omb1 = (float)(1.0 - a.beta1);
    c.omb2 = (float)(1.0 - a.beta2);
    c.eps = a.eps;
    return c;
}

// The SH coefficients (as given) of the visible rows: one warp per row, lane k
// updating coefficients k, k + 32, ... (coalesced), the visible test uniform over
// the warp.
__global__ void adam_sh_kernel(fgs_adam_args a, const uint8_t* __restrict__ flag, const int* __restrict__ step)
{
    const AdamCoef c = adam_coef(a, *step);
    const float ss = (float)(a.lr[1] / c.bc1);
    const int F = 3 * a.M, lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < a.P; i += nwarps) {
        if (!flag[i]) continue;
        for (int k = lane; k < F; k += 32) {
            const size_t j = (size_t)F * i + k;
            adam_update(a.shs[j], a.m_shs[j], a.v_shs[j], a.g_shs[j], c.b1, c.omb1, c.b2, c.omb2, ss, c.bc2s,
                        c.eps);
        }
    }
}

// Everything but the SH coefficients, one thread per row.
__global__ void adam_kernel(fgs_adam_args a, const uint8_t* __restrict__ flag, const int* __restrict__ step)
{
    const AdamCoef c = adam_coef(a, *step);
    const double bc1 = c.bc1;
    const float bc2s = c.bc2s, b1 = c.b1, b2 = c.b2, omb1 = c.omb1, omb2 = c.omb2, eps = c.eps;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.P; i += gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        // means (as given)
        {
            const float ss = (float)(a.lr[0] / bc1);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const size_t j = 3 * (size_t)i + k;
                adam_update(a.xyz[j], a.m_xyz[j], a.v_xyz[j], a.g_xyz[j], b1, omb1, b2, omb2, ss, bc2s, eps);
            }
        }
        // opacity: d/dlogit = d/dopacity * s (1 - s)
        {
            const float ss = (float)(a.lr[2] / bc1);
            const float s = a.opac[i];
            const float g = a.g_opac[i] * (s * (1.f - s));
            adam_update(a.opac_logit[i], a.m_opac[i], a.v_opac[i], g, b1, omb1, b2, omb2, ss, bc2s, eps);
            a.opac[i] = sigmoidf(a.opac_logit[i]);
        }
        // scale: d/dlog = d/dscale * scale
        {
            const float ss = (float)(a.lr[3] / bc1);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const size_t j = 3 * (size_t)i + k;
                const float g = a.g_scale[j] * a.scale[j];
                adam_update(a.log_scale[j], a.m_scale[j], a.v_scale[j], g, b1, omb1, b2, omb2, ss, bc2s, eps);
                a.scale[j] = expf(a.log_scale[j]);
            }
        }
        // rotation: d/dq = (d/dq_hat - q_hat (q_hat . d/dq_hat)) / |q|
        {
            const float ss = (float)(a.lr[4] / bc1);
            float q[4], qh[4], gq[4];
            float n2 = 0.f, dot = 0.f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                q[k] = a.rot_raw[4 * (size_t)i + k];
                n2 += q[k] * q[k];
            }
            const float n = fmaxf(sqrtf(n2), 1e-12f);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                qh[k] = a.rot[4 * (size_t)i + k];
                dot += qh[k] * a.g_rot[4 * (size_t)i + k];
            }
#pragma unroll
            for (int k = 0; k < 4; k++) gq[k] = (a.g_rot[4 * (size_t)i + k] - qh[k] * dot) / n;
            float m2 = 0.f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const size_t j = 4 * (size_t)i + k;
                adam_update(a.rot_raw[j], a.m_rot[j], a.v_rot[j], gq[k], b1, omb1, b2, omb2, ss, bc2s, eps);
                m2 += a.rot_raw[j] * a.rot_raw[j];
            }
            const float nn = fmaxf(sqrtf(m2), 1e-12f);
#pragma unroll
            for (int k = 0; k < 4; k++) a.rot[4 * (size_t)i + k] = a.rot_raw[4 * (size_t)i + k] / nn;
        }
    }
}

__global__ void step_tick_kernel(int* step) { *step += 1; }

namespace {
Window make_window()
{
    // loss.py:7-10: exp(-(x - 5)^2 / (2 * 1.5^2)) in double, stored as float32, normalised in float32
    Window w;
    float sum = 0.f;
    for (int i = 0; i < kWin; i++) {
        w.g[i] = (float)std::exp(-(double)((i - kWin / 2) * (i - kWin / 2)) / (2.0 * 1.5 * 1.5));
        sum += w.g[i];
    }
    for (int i = 0; i < kWin; i++) w.g[i] = w.g[i] / sum;
    return w;
}
}  // namespace

}  // namespace fgs

using namespace fgs;

extern "C" {

size_t fgs_loss_scratch_bytes(int width, int height)
{
    if (width <= kHalo || height <= kHalo) return 0;
    const size_t Wo = (size_t)width - kHalo, Ho = (size_t)height - kHalo;
    const size_t nso = 3 * ((Wo + kTX - 1) / kTX) * ((Ho + kTY - 1) / kTY);
    const size_t nl1 = 3 * (((size_t)width + kTX - 1) / kTX) * (((size_t)height + kTY - 1) / kTY);
    return sizeof(float) * (9 * Wo * Ho + nso + nl1) + 256;
}

int fgs_loss_l1_ssim(int width, int height, const float* pred, const float* target, float* dL_dpred,
                     float l1_grad_scale, float ssim_grad_scale, double* sums, void* scratch, void* stream)
{
    if (width <= kHalo || height <= kHalo || !pred || !target || !dL_dpred || !sums || !scratch) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int Wo = width - kHalo, Ho = height - kHalo;
    float* gmap = static_cast<float*>(scratch);
    const dim3 go((Wo + kTX - 1) / kTX, (Ho + kTY - 1) / kTY, 3);
    const dim3 gp((width + kTX - 1) / kTX, (height + kTY - 1) / kTY, 3);
    float* sp = gmap + (size_t)9 * Wo * Ho;
    float* l1p = sp + (size_t)go.x * go.y * go.z;
    static const Window win = make_window();
    ssim_forward_kernel<<<go, kLossThreads, 0, s>>>(width, height, pred, target, win, ssim_grad_scale, gmap, sp);
    loss_grad_kernel<<<gp, kLossThreads, 0, s>>>(width, height, pred, target, win, gmap, l1_grad_scale, dL_dpred,
                                                 l1p);
    loss_reduce_kernel<<<1, 1024, 0, s>>>(l1p, (int)(gp.x * gp.y * gp.z), sp, (int)(go.x * go.y * go.z), sums);
    note_launches(3);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

int fgs_train_activate(int P, const float* log_scale, const float* rot_raw, const float* opac_logit, float* scale,
                       float* rot, float* opac, void* stream)
{
    if (P < 0 || (P > 0 && (!log_scale || !rot_raw || !opac_logit || !scale || !rot || !opac))) return FGS_ERR_ARG;
    if (P == 0) return FGS_OK;
    activate_kernel<<<(P + 255) / 256 < 4096 ? (P + 255) / 256 : 4096, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        P, log_scale, rot_raw, opac_logit, scale, rot, opac);
    note_launches(1);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

int fgs_densify_dense(int P, const int* radii, const float* dL_dmeans2D, float* grad_sum, int* vis_count,
                      unsigned char* flag, void* stream)
{
    if (P < 0 || (P > 0 && (!radii || !dL_dmeans2D || !grad_sum || !vis_count || !flag))) return FGS_ERR_ARG;
    if (P == 0) return FGS_OK;
    densify_dense_kernel<<<(P + 255) / 256 < 4096 ? (P + 255) / 256 : 4096, 256, 0,
                           static_cast<cudaStream_t>(stream)>>>(P, radii, dL_dmeans2D, grad_sum, vis_count, flag);
    note_launches(1);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

int fgs_adam_step(const fgs_adam_args* a, const unsigned char* flag, int* step, void* stream)
{
    if (!a || !flag || !step || a->P < 0 || a->M < 0) return FGS_ERR_ARG;
    if (!a->xyz || !a->opac_logit || !a->log_scale || !a->rot_raw || !a->opac || !a->scale || !a->rot) return FGS_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    step_tick_kernel<<<1, 1, 0, s>>>(step);
    int n = 1;
    if (a->P > 0) {
        adam_kernel<<<(a->P + 255) / 256 < 4096 ? (a->P + 255) / 256 : 4096, 256, 0, s>>>(*a, flag, step);
        n++;
        if (a->shs && a->M > 0) {
            adam_sh_kernel<<<(a->P + 7) / 8 < 4096 ? (a->P + 7) / 8 : 4096, 256, 0, s>>>(*a, flag, step);
            n++;
        }
    }
    note_launches(n);
    return cudaGetLastError() == cudaSuccess ? FGS_OK : FGS_ERR_CUDA;
}

}  // extern "C"
