/*
 * CPU oracle for the FilterGS rasterizer hot path.  TEST INFRASTRUCTURE ONLY:
 * the product never links or calls this file; tests, the smoke check and the
 * CPU-baseline leg of bench.py use it as the checker.
 *
 * A plain-C restatement of the reference algorithm, compiled twice: once with
 * REAL=float (the FP32 oracle, same expression order as the reference CUDA) and
 * once with REAL=double (the FP64 evaluation of the same splat equations used
 * for the finite-difference check and the FP32-vs-FP64 error report).  In the
 * forward preprocess (cov3D, the view transform, the EWA projection, det, SH
 * colour) the FP32 build also fuses the products the reference build fuses
 * (FMA below), so those outputs equal that build's bit for bit.
 *
 * Reference anchors (paths inside the reference project):
 *   preprocess + OGFS radius ..... antialias/cuda_rasterizer/forward.cu:266-401
 *   cov3D / cov2D / SH colour .... forward.cu:48-185
 *   3-sigma compute_radius ....... forward.cu:187-263 ; FilterGS/cuda/compute_radius_kernel_v2.cu:180-229
 *   in_frustum / ndc2Pix / getRect auxiliary.h:41-56,139-164
 *   duplicate / sort / ranges .... antialias/cuda_rasterizer/rasterizer_impl.cu:78-194,363-445
 *   render forward ............... forward.cu:406-567
 *   render backward .............. backward.cu:399-557
 *   cov2D / preprocess backward .. backward.cu:20-396
 *   LoD visibility mask .......... FilterGS/cuda/compute_radius_kernel_v2.cu:109-169,231-353
 *   LoG cut traversal ............ LoG/model/tensor_tree.py:133-187
 *   ancestor_path builder ........ apps/ancestor.py:21-73
 *   KPC/GTC statistics ........... rasterizer_impl.cu:450-556
 *
 * Parity pins: the FP32 restatement is checked against fixtures produced by
 * the reference's own CUDA build and its torch math (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL float
#endif

#ifdef ORC_F64
#define SFX(name) name##_f64
#define EXPR(x) exp(x)
#define LOGR(x) log(x)
#define SQRTR(x) sqrt(x)
#define POWR(a, b) pow(a, b)
#define CEILR(x) ceil(x)
#define FMAXR(a, b) fmax(a, b)
#define FMINR(a, b) fmin(a, b)
#define LIT(x) ((double)(x))
#define FMA(a, b, c) fma(a, b, c)
#else
#define SFX(name) name##_f32
#define EXPR(x) expf(x)
#define LOGR(x) logf(x)
#define SQRTR(x) sqrtf(x)
#define POWR(a, b) powf(a, b)
#define CEILR(x) ceilf(x)
#define FMAXR(a, b) fmaxf(a, b)
#define FMINR(a, b) fminf(a, b)
#define LIT(x) ((float)(x))
#define FMA(a, b, c) fmaf(a, b, c)
#endif

/* The reference's binning tile (config.h:16-17).  A build with other -DBLOCK_X /
   -DBLOCK_Y serves the tile-shape study of tests/test_tile_shape_cpu.py only;
   OGFS_LAMBDA_PIXELS is lambda_G's exponent (BLOCK_X*BLOCK_Y in the reference,
   forward.cu:348), which that study keeps at 256 while the tile changes. */
#ifndef BLOCK_X
#define BLOCK_X 16
#endif
#ifndef BLOCK_Y
#define BLOCK_Y 16
#endif
#ifndef OGFS_LAMBDA_PIXELS
#define OGFS_LAMBDA_PIXELS (BLOCK_X * BLOCK_Y)
#endif
#define BLOCK_SIZE (BLOCK_X * BLOCK_Y)

typedef REAL real;

/* ---------------------------------------------------------------- helpers */

static inline real rmin(real a, real b) { return a < b ? a : b; }
static inline real rmax(real a, real b) { return a > b ? a : b; }

/* auxiliary.h:41-44 -- evaluated in double precision, as the reference's
 * double literals promote it. */
static inline real ndc2pix(real v, int S) { return (real)((((double)v + 1.0) * S - 1.0) * 0.5); }

/* auxiliary.h:46-56 -- float division, truncation toward zero. */
static inline void get_rect(real px, real py, int r, int gx, int gy, int tx, int ty,
                            int *xmin, int *ymin, int *xmax, int *ymax)
{
    int a = (int)((px - r) / tx), b = (int)((py - r) / ty);
    int c = (int)((px + r + tx - 1) / tx), d = (int)((py + r + ty - 1) / ty);
    a = a < 0 ? 0 : a; b = b < 0 ? 0 : b; c = c < 0 ? 0 : c; d = d < 0 ? 0 : d;
    *xmin = a > gx ? gx : a; *ymin = b > gy ? gy : b;
    *xmax = c > gx ? gx : c; *ymax = d > gy ? gy : d;
}

/* column-major 4x4 matrices as stored by the reference (auxiliary.h:58-106) */
static inline void xform4x3(const real *p, const real *m, real *o)
{
    o[0] = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
    o[1] = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
    o[2] = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
}
static inline void xform4x4(const real *p, const real *m, real *o)
{
    xform4x3(p, m, o);
    o[3] = m[3] * p[0] + m[7] * p[1] + m[11] * p[2] + m[15];
}

/* 3x3 matrices stored column-major: a[c][r] (the glm convention the
 * reference's covariance code is written in). */
typedef struct { real m[3][3]; } m3;
static inline m3 m3_mul(const m3 *a, const m3 *b)
{
    m3 r;
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++)
            r.m[c][k] = a->m[0][k] * b->m[c][0] + a->m[1][k] * b->m[c][1] + a->m[2][k] * b->m[c][2];
    return r;
}
static inline m3 m3_t(const m3 *a)
{
    m3 r;
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++) r.m[c][k] = a->m[k][c];
    return r;
}

/* forward.cu:151-185 (quaternion used as given, not normalised) */
static void cov3d_from(const real *s, real mod, const real *q, real *cov)
{
    m3 S = {{{0}}}, R;
    S.m[0][0] = mod * s[0]; S.m[1][1] = mod * s[1]; S.m[2][2] = mod * s[2];
    real r = q[0], x = q[1], y = q[2], z = q[3];
    R.m[0][0] = 1 - 2 * (y * y + z * z); R.m[0][1] = 2 * (x * y - r * z); R.m[0][2] = 2 * (x * z + r * y);
    R.m[1][0] = 2 * (x * y + r * z); R.m[1][1] = 1 - 2 * (x * x + z * z); R.m[1][2] = 2 * (y * z - r * x);
    R.m[2][0] = 2 * (x * z - r * y); R.m[2][1] = 2 * (y * z + r * x); R.m[2][2] = 1 - 2 * (x * x + y * y);
    m3 M = m3_mul(&S, &R);
    m3 Mt = m3_t(&M);
    m3 Sig = m3_mul(&Mt, &M);
    cov[0] = Sig.m[0][0]; cov[1] = Sig.m[0][1]; cov[2] = Sig.m[0][2];
    cov[3] = Sig.m[1][1]; cov[4] = Sig.m[1][2]; cov[5] = Sig.m[2][2];
}

/* The forward preprocess's covariance chain and view transform with the
 * multiply-add grouping of the reference build (nvcc fuses a product into the
 * add that consumes it; which one was found by comparing candidate groupings
 * with the reference build's cov3D, conic and colour bits on three 1080p views
 * of a 2M-Gaussian scene).  dot3r: ((a0 b0 + a1 b1) + a2 b2) with the first and
 * last products fused. */
static inline real dot3r(real a0, real b0, real a1, real b1, real a2, real b2)
{
    return FMA(a2, b2, FMA(a0, b0, a1 * b1));
}
static inline void xform4x3_ref(const real *p, const real *m, real *o)
{
    for (int r = 0; r < 3; r++) o[r] = dot3r(m[r], p[0], m[4 + r], p[1], m[8 + r], p[2]) + m[12 + r];
}
static inline void xform4x4_ref(const real *p, const real *m, real *o)
{
    for (int r = 0; r < 4; r++) o[r] = dot3r(m[r], p[0], m[4 + r], p[1], m[8 + r], p[2]) + m[12 + r];
}

/* forward.cu:151-185 in the reference build's grouping: y y + z z unfused, the
 * entries that share x z fuse r y, the others fuse their first product. */
static void cov3d_ref(const real *s, real mod, const real *q, real *cov)
{
    const real r = q[0], x = q[1], y = q[2], z = q[3];
    real R[3][3];
    R[0][0] = 1 - 2 * (y * y + z * z);
    R[0][1] = 2 * FMA(x, y, -(r * z));
    R[0][2] = 2 * FMA(r, y, x * z);
    R[1][0] = 2 * FMA(x, y, r * z);
    R[1][1] = 1 - 2 * FMA(x, x, z * z);
    R[1][2] = 2 * FMA(y, z, -(r * x));
    R[2][0] = 2 * FMA(-r, y, x * z);
    R[2][1] = 2 * FMA(y, z, r * x);
    R[2][2] = 1 - 2 * FMA(x, x, y * y);
    const real sc[3] = {mod * s[0], mod * s[1], mod * s[2]};
    real M[3][3];
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++) M[c][k] = sc[k] * R[c][k];
#define SIG(c, k) dot3r(M[k][0], M[c][0], M[k][1], M[c][1], M[k][2], M[c][2])
    cov[0] = SIG(0, 0); cov[1] = SIG(0, 1); cov[2] = SIG(0, 2);
    cov[3] = SIG(1, 1); cov[4] = SIG(1, 2); cov[5] = SIG(2, 2);
#undef SIG
}

/* forward.cu:102-146 in the reference build's grouping (every dot fuses its
 * first and last product; W J fuses its J[2] term). */
static void ewa_ref(const real *mean, real fx, real fy, real tanx, real tany, const real *cov3D, const real *v,
                    real *c00, real *c01, real *c11)
{
    real t[3];
    xform4x3_ref(mean, v, t);
    const real limx = LIT(1.3) * tanx, limy = LIT(1.3) * tany;
    t[0] = rmin(limx, rmax(-limx, t[0] / t[2])) * t[2];
    t[1] = rmin(limy, rmax(-limy, t[1] / t[2])) * t[2];
    const real tz2 = t[2] * t[2];
    const real j00 = fx / t[2], j02 = -(fx * t[0]) / tz2, j11 = fy / t[2], j12 = -(fy * t[1]) / tz2;
    real T[2][3];
    for (int k = 0; k < 3; k++) {
        T[0][k] = FMA(v[4 * k + 2], j02, v[4 * k] * j00);
        T[1][k] = FMA(v[4 * k + 2], j12, v[4 * k + 1] * j11);
    }
    const real V[3][3] = {{cov3D[0], cov3D[1], cov3D[2]}, {cov3D[1], cov3D[3], cov3D[4]},
                          {cov3D[2], cov3D[4], cov3D[5]}};
    real X[3][2];
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 2; k++) X[c][k] = dot3r(T[k][0], V[0][c], T[k][1], V[1][c], T[k][2], V[2][c]);
#define CV(c, k) dot3r(X[0][k], T[c][0], X[1][k], T[c][1], X[2][k], T[c][2])
    *c00 = CV(0, 0); *c01 = CV(0, 1); *c11 = CV(1, 1);
#undef CV
}

/* EWA projection shared by forward, backward and the radius kernels
 * (forward.cu:102-146, backward.cu:166-194).  Fills T (= W*J) and the
 * clamp flags; returns the un-dilated 2D covariance. */
typedef struct { m3 T, W; real t[3]; real J00, J02, J11, J12; int xclamp, yclamp; real txtz, tytz; } ewa_t;

static void ewa(const real *mean, real fx, real fy, real tanx, real tany, const real *cov3D,
                const real *view, ewa_t *e, real *c00, real *c01, real *c11)
{
    real t[3];
    xform4x3(mean, view, t);
    const real limx = LIT(1.3) * tanx, limy = LIT(1.3) * tany;
    const real txtz = t[0] / t[2], tytz = t[1] / t[2];
    e->xclamp = txtz < -limx || txtz > limx;
    e->yclamp = tytz < -limy || tytz > limy;
    e->txtz = txtz; e->tytz = tytz;
    t[0] = rmin(limx, rmax(-limx, txtz)) * t[2];
    t[1] = rmin(limy, rmax(-limy, tytz)) * t[2];
    e->t[0] = t[0]; e->t[1] = t[1]; e->t[2] = t[2];
    m3 J = {{{0}}};
    J.m[0][0] = fx / t[2]; J.m[0][1] = 0; J.m[0][2] = -(fx * t[0]) / (t[2] * t[2]);
    J.m[1][0] = 0; J.m[1][1] = fy / t[2]; J.m[1][2] = -(fy * t[1]) / (t[2] * t[2]);
    e->J00 = J.m[0][0]; e->J02 = J.m[0][2]; e->J11 = J.m[1][1]; e->J12 = J.m[1][2];
    m3 W;
    W.m[0][0] = view[0]; W.m[0][1] = view[4]; W.m[0][2] = view[8];
    W.m[1][0] = view[1]; W.m[1][1] = view[5]; W.m[1][2] = view[9];
    W.m[2][0] = view[2]; W.m[2][1] = view[6]; W.m[2][2] = view[10];
    e->W = W;
    m3 T = m3_mul(&W, &J);
    e->T = T;
    m3 V;
    V.m[0][0] = cov3D[0]; V.m[0][1] = cov3D[1]; V.m[0][2] = cov3D[2];
    V.m[1][0] = cov3D[1]; V.m[1][1] = cov3D[3]; V.m[1][2] = cov3D[4];
    V.m[2][0] = cov3D[2]; V.m[2][1] = cov3D[4]; V.m[2][2] = cov3D[5];
    m3 Tt = m3_t(&T), Vt = m3_t(&V);
    m3 A = m3_mul(&Tt, &Vt);
    m3 C = m3_mul(&A, &T);
    *c00 = C.m[0][0]; *c01 = C.m[0][1]; *c11 = C.m[1][1];
}

/* DILATE_PIXEL is a double literal in the reference: max(float, 0.3) runs in
 * double (forward.cu:141-144) and so does "+= 0.3" (backward.cu:197-199). */
static inline real dil_max(real c) { return (real)((double)c > 0.3 ? (double)c : 0.3); }
static inline real dil_add(real c) { return (real)((double)c + 0.3); }

static const double SH_C0 = 0.28209479177387814;
static const double SH_C1 = 0.4886025119029199;
static const double SH_C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                                -1.0925484305920792, 0.5462742152960396};
static const double SH_C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                                0.3731763325901154, -0.4570457994644658, 1.445305721320277,
                                -0.5900435899266435};

/* forward.cu:48-99 */
/* forward.cu:48-99 in the reference build's grouping: |dir|^2 like dot3r,
 * C0 sh0 - C1 y sh1 fuses C1 y sh1, each later term fuses its final product with
 * the coefficient into the running sum, 3 xx - yy, xx - 3 yy and
 * (2 zz - 3 xx) - 3 yy fuse the product by 3. */
static void sh_to_rgb(int deg, int M, const real *pos, const real *campos, const real *sh_all, int idx,
                      real *rgb, uint8_t *clamped)
{
    const real c0 = (real)SH_C0, c1 = (real)SH_C1;
    real dir[3] = {pos[0] - campos[0], pos[1] - campos[1], pos[2] - campos[2]};
    real len = SQRTR(dot3r(dir[0], dir[0], dir[1], dir[1], dir[2], dir[2]));
    dir[0] = dir[0] / len; dir[1] = dir[1] / len; dir[2] = dir[2] / len;
    const real *sh = sh_all + (size_t)idx * M * 3;
    real x = dir[0], y = dir[1], z = dir[2];
    real xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    real f[5] = {(real)SH_C2[0] * xy, (real)SH_C2[1] * yz, (real)SH_C2[2] * (LIT(2.0) * zz - xx - yy),
                 (real)SH_C2[3] * xz, (real)SH_C2[4] * (xx - yy)};
    real q4 = LIT(4.0) * zz - xx - yy;
    real g[7] = {(real)SH_C3[0] * y * FMA(LIT(3.0), xx, -yy), (real)SH_C3[1] * xy * z, (real)SH_C3[2] * y * q4,
                 (real)SH_C3[3] * z * FMA(LIT(-3.0), yy, FMA(LIT(-3.0), xx, LIT(2.0) * zz)),
                 (real)SH_C3[4] * x * q4, (real)SH_C3[5] * z * (xx - yy),
                 (real)SH_C3[6] * x * FMA(LIT(-3.0), yy, xx)};
    for (int ch = 0; ch < 3; ch++) {
#define S(k) sh[(k) * 3 + ch]
        real res = c0 * S(0);
        if (deg > 0) {
            res = FMA(-(c1 * y), S(1), res);
            res = FMA(c1 * z, S(2), res);
            res = FMA(-(c1 * x), S(3), res);
            if (deg > 1) {
                for (int i = 0; i < 5; i++) res = FMA(f[i], S(4 + i), res);
                if (deg > 2)
                    for (int i = 0; i < 7; i++) res = FMA(g[i], S(9 + i), res);
            }
        }
#undef S
        res += LIT(0.5);
        clamped[3 * idx + ch] = res < 0;
        rgb[3 * idx + ch] = res < 0 ? 0 : res;
    }
}

/* ---------------------------------------------------------------- preprocess */

typedef struct {
    int P, D, M, W, H;
    const real *means, *scales, *rots, *opac, *shs, *cov3D_precomp, *colors_precomp;
    const real *view, *proj, *campos;
    real scale_mod, tanx, tany;
    int use_filter;
    real eps_scale, eps_max, energy_floor, ratio_min;
    real filter3d; /* 3D filter: cov3D += (filter3d * z_view / focal_x)^2 I ; 0 = off */
} SFX(orc_pre_args);

/* forward.cu:266-401.  Outputs are dense [P] arrays zero-initialised here. */
void SFX(orc_preprocess)(const SFX(orc_pre_args) * a, int *radii, real *means2D, real *depths,
                         real *conic_o, real *rgb, uint8_t *clamped, uint32_t *tiles, real *cov3D_out)
{
    const int P = a->P;
    const real fy = a->H / (LIT(2.0) * a->tany), fx = a->W / (LIT(2.0) * a->tanx);
    const int gx = (a->W + BLOCK_X - 1) / BLOCK_X, gy = (a->H + BLOCK_Y - 1) / BLOCK_Y;
    /* lambda_G (forward.cu:346-351); OGFS_LAMBDA_PIXELS = 256 = BLOCK_X*BLOCK_Y of the reference. */
    const real eps_pix = LIT(1.0) / LIT(255.0);
    const real eps_base = FMAXR(LIT(0.0), LIT(1.0) - eps_pix);
    const real lg_raw = LIT(1.0) - POWR(eps_base, (real)(OGFS_LAMBDA_PIXELS));
    real lg = eps_pix + a->eps_scale * (lg_raw - eps_pix);
    lg = FMINR(FMAXR(lg, eps_pix), a->eps_max);
    const real log_lg = LOGR(lg);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P; i++) {
        radii[i] = 0; tiles[i] = 0; depths[i] = 0;
        means2D[2 * i] = means2D[2 * i + 1] = 0;
        conic_o[4 * i] = conic_o[4 * i + 1] = conic_o[4 * i + 2] = conic_o[4 * i + 3] = 0;
        const real *p = a->means + 3 * (size_t)i;
        real ph[4], pv[3];
        xform4x4_ref(p, a->proj, ph);
        real pw = LIT(1.0) / (ph[3] + LIT(0.0000001));
        real pp[3] = {ph[0] * pw, ph[1] * pw, ph[2] * pw};
        xform4x3_ref(p, a->view, pv);
        if (pv[2] <= LIT(0.2)) continue; /* auxiliary.h:154 */
        real cov[6];
        if (a->cov3D_precomp) memcpy(cov, a->cov3D_precomp + 6 * (size_t)i, sizeof(cov));
        else cov3d_ref(a->scales + 3 * (size_t)i, a->scale_mod, a->rots + 4 * (size_t)i, cov);
        if (a->filter3d > 0) {
            real sf = a->filter3d * pv[2] / fx;
            real v = sf * sf;
            cov[0] += v; cov[3] += v; cov[5] += v;
        }
        if (cov3D_out) memcpy(cov3D_out + 6 * (size_t)i, cov, sizeof(cov));
        real c00, c01, c11;
        ewa_ref(p, fx, fy, a->tanx, a->tany, cov, a->view, &c00, &c01, &c11);
        if (a->use_filter) { c00 = dil_max(c00); c11 = dil_max(c11); }
        real det = FMA(c00, c11, -(c01 * c01));
        if (det == LIT(0.0)) continue;
        real dinv = LIT(1.0) / det;
        real con[3] = {c11 * dinv, -c01 * dinv, c00 * dinv};
        real op = FMAXR(a->opac[i], LIT(1e-6));
        real energy = FMAXR(LOGR(op) - log_lg, a->energy_floor);
        real mid = LIT(0.5) * (c00 + c11);
        real sd = SQRTR(FMAXR(LIT(0.0), mid * mid - det));
        real l1 = mid + sd, l2 = mid - sd;
        real lmax = FMAXR(FMAXR(l1, l2), LIT(1e-6));
        real rb = LIT(3.0) * SQRTR(lmax);
        real rm = SQRTR(LIT(2.0) * energy * lmax);
        rm = FMINR(rm, rb);
        rm = FMAXR(rm, a->ratio_min * rb);
        int rpx = (int)CEILR(rm + LIT(1.0));
        if (rpx < 1) rpx = 1;
        real px = ndc2pix(pp[0], a->W), py = ndc2pix(pp[1], a->H);
        int x0, y0, x1, y1;
        get_rect(px, py, rpx, gx, gy, BLOCK_X, BLOCK_Y, &x0, &y0, &x1, &y1);
        int ext = (x1 - x0) * (y1 - y0);
        if (ext == 0) continue;
        if (!a->colors_precomp && a->shs) sh_to_rgb(a->D, a->M, p, a->campos, a->shs, i, rgb, clamped);
        depths[i] = pv[2];
        radii[i] = rpx;
        means2D[2 * i] = px; means2D[2 * i + 1] = py;
        conic_o[4 * i] = con[0]; conic_o[4 * i + 1] = con[1]; conic_o[4 * i + 2] = con[2]; conic_o[4 * i + 3] = op;
        tiles[i] = (uint32_t)ext;
    }
}

/* forward.cu:187-263 (antialias _C.compute_radius: z>0.2 and +-1.3 NDC cull,
 * no dilation).  variant 1 = FilterGS/LoG v2 kernel (compute_radius_kernel_v2.cu:180-229:
 * +-1.3 NDC only, diagonal max 0.3). */
void SFX(orc_compute_radius)(int variant, int P, const real *means, const real *scales, const real *rots,
                             const real *view, const real *proj, real fx, real fy, real tanx, real tany,
                             real *radius)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P; i++) {
        radius[i] = 0;
        const real *p = means + 3 * (size_t)i;
        real ph[4], pv[3];
        xform4x4(p, proj, ph);
        real pw = LIT(1.0) / (ph[3] + LIT(0.0000001));
        real pp[2] = {ph[0] * pw, ph[1] * pw};
        xform4x3(p, view, pv);
        if (variant == 0 && pv[2] <= LIT(0.2)) continue;
        if ((double)pp[0] < -1.3 || (double)pp[0] > 1.3 || (double)pp[1] < -1.3 || (double)pp[1] > 1.3) continue;
        real cov[6];
        cov3d_from(scales + 3 * (size_t)i, LIT(1.0), rots + 4 * (size_t)i, cov);
        ewa_t e;
        real c00, c01, c11;
        ewa(p, fx, fy, tanx, tany, cov, view, &e, &c00, &c01, &c11);
        if (variant == 1) { c00 = dil_max(c00); c11 = dil_max(c11); }
        real det = c00 * c11 - c01 * c01;
        if (det == LIT(0.0)) continue;
        real mid = LIT(0.5) * (c00 + c11);
        real l1 = mid + SQRTR(FMAXR(LIT(0.1), mid * mid - det));
        real l2 = mid - SQRTR(FMAXR(LIT(0.1), mid * mid - det));
        radius[i] = LIT(3.0) * SQRTR(FMAXR(l1, l2));
    }
}

/* rasterizer_impl.cu:97-109 + auxiliary.h:139-164 */
void SFX(orc_mark_visible)(int P, const real *means, const real *view, uint8_t *present)
{
    for (int i = 0; i < P; i++) {
        real pv[3];
        xform4x3(means + 3 * (size_t)i, view, pv);
        present[i] = pv[2] > LIT(0.2);
    }
}

/* ---------------------------------------------------------------- binning */

typedef struct { uint64_t key; uint32_t val; uint32_t seq; } kv_t;
static int kv_cmp(const void *x, const void *y)
{
    const kv_t *a = x, *b = y;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->seq < b->seq ? -1 : (a->seq > b->seq);
}

/* rasterizer_impl.cu:113-147 (duplicateWithKeys), :427-445 (stable sort over
 * the low 32+bit key bits, tile ranges).  Returns K.  keys/vals must hold the
 * count returned by orc_count_pairs. */
static uint32_t float_bits(real d) { float f = (float)d; uint32_t u; memcpy(&u, &f, 4); return u; }

long long SFX(orc_count_pairs)(int P, const uint32_t *tiles)
{
    long long k = 0;
    for (int i = 0; i < P; i++) k += tiles[i];
    return k;
}

long long SFX(orc_bin)(int P, int W, int H, const int *radii, const real *means2D, const real *depths,
                       uint64_t *keys, uint32_t *vals, uint32_t *ranges)
{
    const int gx = (W + BLOCK_X - 1) / BLOCK_X, gy = (H + BLOCK_Y - 1) / BLOCK_Y;
    long long n = 0;
    for (int i = 0; i < P; i++) {
        if (radii[i] <= 0) continue;
        int x0, y0, x1, y1;
        get_rect(means2D[2 * i], means2D[2 * i + 1], radii[i], gx, gy, BLOCK_X, BLOCK_Y, &x0, &y0, &x1, &y1);
        n += (long long)(x1 - x0) * (y1 - y0);
    }
    kv_t *kv = malloc(sizeof(kv_t) * (n > 0 ? n : 1));
    long long o = 0;
    for (int i = 0; i < P; i++) {
        if (radii[i] <= 0) continue;
        int x0, y0, x1, y1;
        get_rect(means2D[2 * i], means2D[2 * i + 1], radii[i], gx, gy, BLOCK_X, BLOCK_Y, &x0, &y0, &x1, &y1);
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) {
                kv[o].key = ((uint64_t)(uint32_t)(y * gx + x) << 32) | float_bits(depths[i]);
                kv[o].val = (uint32_t)i;
                kv[o].seq = (uint32_t)o;
                o++;
            }
    }
    qsort(kv, n, sizeof(kv_t), kv_cmp);
    memset(ranges, 0, sizeof(uint32_t) * 2 * gx * gy);
    for (long long k = 0; k < n; k++) {
        keys[k] = kv[k].key;
        vals[k] = kv[k].val;
        uint32_t t = (uint32_t)(kv[k].key >> 32);
        if (k == 0 || (uint32_t)(kv[k - 1].key >> 32) != t) ranges[2 * t] = (uint32_t)k;
        if (k == n - 1 || (uint32_t)(kv[k + 1].key >> 32) != t) ranges[2 * t + 1] = (uint32_t)(k + 1);
    }
    free(kv);
    return n;
}

/* ---------------------------------------------------------------- render forward */

static inline void atomic_max_real(real *addr, real v)
{
#ifdef ORC_F64
    uint64_t *p = (uint64_t *)addr, old = __atomic_load_n(p, __ATOMIC_RELAXED);
    for (;;) {
        double cur; memcpy(&cur, &old, 8);
        if (!(v > cur)) return;
        uint64_t nw; memcpy(&nw, &v, 8);
        if (__atomic_compare_exchange_n(p, &old, nw, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
    }
#else
    uint32_t *p = (uint32_t *)addr, old = __atomic_load_n(p, __ATOMIC_RELAXED);
    for (;;) {
        float cur; memcpy(&cur, &old, 4);
        if (!(v > cur)) return;
        uint32_t nw; memcpy(&nw, &v, 4);
        if (__atomic_compare_exchange_n(p, &old, nw, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return;
    }
#endif
}

/* forward.cu:406-567.  kv_sum/kv_cnt (optional) are the per-pair statistics
 * of forward.cu:532-540.  out_point_weight is an exact max here (the
 * reference's is a racy read-compare-write). tile_lo/tile_hi restrict the
 * work to a range of tile indices (CPU-baseline sampling); -1 = all. */
void SFX(orc_render)(int W, int H, const uint32_t *ranges, const uint32_t *vals, const real *means2D,
                     const real *feat, const real *conic_o, const real *bg, real *out_color, real *final_T,
                     uint32_t *n_contrib, int *point_id, real *pw_pixel, real *point_weight, real *kv_sum,
                     uint32_t *kv_cnt, int tile_lo, int tile_hi)
{
    const int gx = (W + BLOCK_X - 1) / BLOCK_X, gy = (H + BLOCK_Y - 1) / BLOCK_Y;
    if (tile_lo < 0) { tile_lo = 0; tile_hi = gx * gy; }
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = tile_lo; t < tile_hi; t++) {
        const int bx = t % gx, by = t / gx;
        const uint32_t r0 = ranges[2 * t], r1 = ranges[2 * t + 1];
        for (int ly = 0; ly < BLOCK_Y; ly++)
            for (int lx = 0; lx < BLOCK_X; lx++) {
                const int x = bx * BLOCK_X + lx, y = by * BLOCK_Y + ly;
                if (x >= W || y >= H) continue;
                const real pxf = (real)x, pyf = (real)y;
                real T = LIT(1.0), C[3] = {0, 0, 0}, wmax = 0;
                uint32_t contributor = 0, last = 0;
                int maxid = -1;
                for (uint32_t k = r0; k < r1; k++) {
                    contributor++;
                    const uint32_t id = vals[k];
                    const real dx = means2D[2 * id] - pxf, dy = means2D[2 * id + 1] - pyf;
                    const real *co = conic_o + 4 * (size_t)id;
                    const real power = LIT(-0.5) * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
                    if (power > LIT(0.0)) continue;
                    const real alpha = rmin(LIT(0.99), co[3] * EXPR(power));
                    if (alpha < LIT(1.0) / LIT(255.0)) continue;
                    const real test_T = T * (1 - alpha);
                    if (test_T < LIT(0.0001)) break;
                    for (int ch = 0; ch < 3; ch++) C[ch] += feat[3 * (size_t)id + ch] * alpha * T;
                    const real w = T * alpha;
                    if (w > wmax) { wmax = w; maxid = (int)id; }
                    atomic_max_real(&point_weight[id], w);
                    if (kv_sum) {
#pragma omp atomic
                        kv_sum[k] += w;
#pragma omp atomic
                        kv_cnt[k] += 1;
                    }
                    T = test_T;
                    last = contributor;
                }
                const int pix = y * W + x;
                final_T[pix] = T;
                n_contrib[pix] = last;
                for (int ch = 0; ch < 3; ch++) out_color[ch * H * W + pix] = C[ch] + T * bg[ch];
                point_id[pix] = maxid;
                pw_pixel[pix] = wmax;
            }
    }
}

/* ---------------------------------------------------------------- render backward */

static inline void atomic_add_real(real *addr, real v)
{
#pragma omp atomic
    *addr += v;
}

/* backward.cu:399-557.  consistent != 0 masks the opacity/G gradient where the
 * forward clamped alpha to 0.99 (the reference does not).  Gradient outputs
 * must be zeroed by the caller; dmean2D is [P,3] (z untouched), dconic [P,4]
 * (x, y, -, w as in the reference's float4 view of [P,2,2]). */
void SFX(orc_render_bwd)(int W, int H, const uint32_t *ranges, const uint32_t *vals, const real *means2D,
                         const real *feat, const real *conic_o, const real *bg, const real *final_T,
                         const uint32_t *n_contrib, const real *dL_dpix, real *dmean2D, real *dconic,
                         real *dopac, real *dcolor, int consistent, int tile_lo, int tile_hi)
{
    const int gx = (W + BLOCK_X - 1) / BLOCK_X, gy = (H + BLOCK_Y - 1) / BLOCK_Y;
    if (tile_lo < 0) { tile_lo = 0; tile_hi = gx * gy; }
    const real ddelx_dx = (real)(0.5 * W), ddely_dy = (real)(0.5 * H);
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = tile_lo; t < tile_hi; t++) {
        const int bx = t % gx, by = t / gx;
        const uint32_t r0 = ranges[2 * t], r1 = ranges[2 * t + 1];
        for (int ly = 0; ly < BLOCK_Y; ly++)
            for (int lx = 0; lx < BLOCK_X; lx++) {
                const int x = bx * BLOCK_X + lx, y = by * BLOCK_Y + ly;
                if (x >= W || y >= H) continue;
                const int pix = y * W + x;
                const real pxf = (real)x, pyf = (real)y;
                const real T_final = final_T[pix];
                real T = T_final;
                const uint32_t last = n_contrib[pix];
                real accum[3] = {0, 0, 0}, last_color[3] = {0, 0, 0}, last_alpha = 0;
                real dpix[3];
                for (int ch = 0; ch < 3; ch++) dpix[ch] = dL_dpix[ch * H * W + pix];
                /* contributor index of entry k (1-based position in the tile list) */
                for (uint32_t k = r1; k-- > r0;) {
                    const uint32_t contributor = k - r0; /* == ref's decremented counter */
                    if (contributor >= last) continue;
                    const uint32_t id = vals[k];
                    const real dx = means2D[2 * id] - pxf, dy = means2D[2 * id + 1] - pyf;
                    const real *co = conic_o + 4 * (size_t)id;
                    const real power = LIT(-0.5) * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
                    if (power > LIT(0.0)) continue;
                    const real G = EXPR(power);
                    const real alpha = rmin(LIT(0.99), co[3] * G);
                    if (alpha < LIT(1.0) / LIT(255.0)) continue;
                    T = T / (LIT(1.0) - alpha);
                    const real dchdc = alpha * T;
                    real dL_dalpha = 0;
                    for (int ch = 0; ch < 3; ch++) {
                        const real c = feat[3 * (size_t)id + ch];
                        accum[ch] = last_alpha * last_color[ch] + (LIT(1.0) - last_alpha) * accum[ch];
                        last_color[ch] = c;
                        dL_dalpha += (c - accum[ch]) * dpix[ch];
                        atomic_add_real(&dcolor[3 * (size_t)id + ch], dchdc * dpix[ch]);
                    }
                    dL_dalpha *= T;
                    last_alpha = alpha;
                    real bgdot = 0;
                    for (int ch = 0; ch < 3; ch++) bgdot += bg[ch] * dpix[ch];
                    dL_dalpha += (-T_final / (LIT(1.0) - alpha)) * bgdot;
                    if (consistent && co[3] * G > LIT(0.99)) dL_dalpha = 0;
                    const real dL_dG = co[3] * dL_dalpha;
                    const real gdx = G * dx, gdy = G * dy;
                    const real dG_ddelx = -gdx * co[0] - gdy * co[1];
                    const real dG_ddely = -gdy * co[2] - gdx * co[1];
                    atomic_add_real(&dmean2D[3 * (size_t)id], dL_dG * dG_ddelx * ddelx_dx);
                    atomic_add_real(&dmean2D[3 * (size_t)id + 1], dL_dG * dG_ddely * ddely_dy);
                    atomic_add_real(&dconic[4 * (size_t)id], LIT(-0.5) * gdx * dx * dL_dG);
                    atomic_add_real(&dconic[4 * (size_t)id + 1], LIT(-0.5) * gdx * dy * dL_dG);
                    atomic_add_real(&dconic[4 * (size_t)id + 3], LIT(-0.5) * gdy * dy * dL_dG);
                    atomic_add_real(&dopac[id], G * dL_dalpha);
                }
            }
    }
}

/* ---------------------------------------------------------------- preprocess backward */

static inline void dnormvdv3(const real *v, const real *dv, real *o)
{
    real s2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    real inv = LIT(1.0) / SQRTR(s2 * s2 * s2);
    o[0] = ((+s2 - v[0] * v[0]) * dv[0] - v[1] * v[0] * dv[1] - v[2] * v[0] * dv[2]) * inv;
    o[1] = (-v[0] * v[1] * dv[0] + (s2 - v[1] * v[1]) * dv[1] - v[2] * v[1] * dv[2]) * inv;
    o[2] = (-v[0] * v[2] * dv[0] - v[1] * v[2] * dv[1] + (s2 - v[2] * v[2]) * dv[2]) * inv;
}

/* backward.cu:20-139 */
static void sh_bwd(int idx, int deg, int M, const real *pos, const real *campos, const real *shs,
                   const uint8_t *clamped, const real *dcolor, real *dmean, real *dsh)
{
    real dir0[3] = {pos[0] - campos[0], pos[1] - campos[1], pos[2] - campos[2]};
    real len = SQRTR(dir0[0] * dir0[0] + dir0[1] * dir0[1] + dir0[2] * dir0[2]);
    real x = dir0[0] / len, y = dir0[1] / len, z = dir0[2] / len;
    const real *sh = shs + (size_t)idx * M * 3;
    real *g = dsh + (size_t)idx * M * 3;
    real dRGB[3];
    for (int c = 0; c < 3; c++) dRGB[c] = clamped[3 * idx + c] ? 0 : dcolor[3 * (size_t)idx + c];
    real dx3[3] = {0, 0, 0}, dy3[3] = {0, 0, 0}, dz3[3] = {0, 0, 0};
    const real c0 = (real)SH_C0, c1 = (real)SH_C1;
    const real C2_0 = (real)SH_C2[0], C2_1 = (real)SH_C2[1], C2_2 = (real)SH_C2[2], C2_3 = (real)SH_C2[3], C2_4 = (real)SH_C2[4];
    const real C3_0 = (real)SH_C3[0], C3_1 = (real)SH_C3[1], C3_2 = (real)SH_C3[2], C3_3 = (real)SH_C3[3],
               C3_4 = (real)SH_C3[4], C3_5 = (real)SH_C3[5], C3_6 = (real)SH_C3[6];
    for (int c = 0; c < 3; c++) {
#define SH(k) sh[(k) * 3 + c]
#define G(k) g[(k) * 3 + c]
        G(0) = c0 * dRGB[c];
        if (deg > 0) {
            G(1) = -c1 * y * dRGB[c]; G(2) = c1 * z * dRGB[c]; G(3) = -c1 * x * dRGB[c];
            dx3[c] = -c1 * SH(3); dy3[c] = -c1 * SH(1); dz3[c] = c1 * SH(2);
            if (deg > 1) {
                real xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
                G(4) = C2_0 * xy * dRGB[c]; G(5) = C2_1 * yz * dRGB[c];
                G(6) = C2_2 * (2 * zz - xx - yy) * dRGB[c]; G(7) = C2_3 * xz * dRGB[c];
                G(8) = C2_4 * (xx - yy) * dRGB[c];
                dx3[c] += C2_0 * y * SH(4) + C2_2 * 2 * -x * SH(6) + C2_3 * z * SH(7) + C2_4 * 2 * x * SH(8);
                dy3[c] += C2_0 * x * SH(4) + C2_1 * z * SH(5) + C2_2 * 2 * -y * SH(6) + C2_4 * 2 * -y * SH(8);
                dz3[c] += C2_1 * y * SH(5) + C2_2 * 2 * 2 * z * SH(6) + C2_3 * x * SH(7);
                if (deg > 2) {
                    G(9) = C3_0 * y * (3 * xx - yy) * dRGB[c]; G(10) = C3_1 * xy * z * dRGB[c];
                    G(11) = C3_2 * y * (4 * zz - xx - yy) * dRGB[c];
                    G(12) = C3_3 * z * (2 * zz - 3 * xx - 3 * yy) * dRGB[c];
                    G(13) = C3_4 * x * (4 * zz - xx - yy) * dRGB[c]; G(14) = C3_5 * z * (xx - yy) * dRGB[c];
                    G(15) = C3_6 * x * (xx - 3 * yy) * dRGB[c];
                    dx3[c] += C3_0 * SH(9) * 3 * 2 * xy + C3_1 * SH(10) * yz + C3_2 * SH(11) * -2 * xy +
                              C3_3 * SH(12) * -3 * 2 * xz + C3_4 * SH(13) * (-3 * xx + 4 * zz - yy) +
                              C3_5 * SH(14) * 2 * xz + C3_6 * SH(15) * 3 * (xx - yy);
                    dy3[c] += C3_0 * SH(9) * 3 * (xx - yy) + C3_1 * SH(10) * xz +
                              C3_2 * SH(11) * (-3 * yy + 4 * zz - xx) + C3_3 * SH(12) * -3 * 2 * yz +
                              C3_4 * SH(13) * -2 * xy + C3_5 * SH(14) * -2 * yz + C3_6 * SH(15) * -3 * 2 * xy;
                    dz3[c] += C3_1 * SH(10) * xy + C3_2 * SH(11) * 4 * 2 * yz +
                              C3_3 * SH(12) * 3 * (2 * zz - xx - yy) + C3_4 * SH(13) * 4 * 2 * xz +
                              C3_5 * SH(14) * (xx - yy);
                }
            }
        }
#undef SH
#undef G
    }
    real ddir[3] = {dx3[0] * dRGB[0] + dx3[1] * dRGB[1] + dx3[2] * dRGB[2],
                    dy3[0] * dRGB[0] + dy3[1] * dRGB[1] + dy3[2] * dRGB[2],
                    dz3[0] * dRGB[0] + dz3[1] * dRGB[1] + dz3[2] * dRGB[2]};
    real dm[3];
    dnormvdv3(dir0, ddir, dm);
    dmean[0] += dm[0]; dmean[1] += dm[1]; dmean[2] += dm[2];
}

/* backward.cu:278-341 (gradient w.r.t. the unnormalised quaternion as used) */
static void cov3d_bwd(const real *scale, real mod, const real *rot, const real *dcov, real *dscale, real *drot)
{
    real r = rot[0], x = rot[1], y = rot[2], z = rot[3];
    m3 R;
    R.m[0][0] = 1 - 2 * (y * y + z * z); R.m[0][1] = 2 * (x * y - r * z); R.m[0][2] = 2 * (x * z + r * y);
    R.m[1][0] = 2 * (x * y + r * z); R.m[1][1] = 1 - 2 * (x * x + z * z); R.m[1][2] = 2 * (y * z - r * x);
    R.m[2][0] = 2 * (x * z - r * y); R.m[2][1] = 2 * (y * z + r * x); R.m[2][2] = 1 - 2 * (x * x + y * y);
    m3 S = {{{0}}};
    real s[3] = {mod * scale[0], mod * scale[1], mod * scale[2]};
    S.m[0][0] = s[0]; S.m[1][1] = s[1]; S.m[2][2] = s[2];
    m3 M = m3_mul(&S, &R);
    m3 dS;
    dS.m[0][0] = dcov[0]; dS.m[0][1] = LIT(0.5) * dcov[1]; dS.m[0][2] = LIT(0.5) * dcov[2];
    dS.m[1][0] = LIT(0.5) * dcov[1]; dS.m[1][1] = dcov[3]; dS.m[1][2] = LIT(0.5) * dcov[4];
    dS.m[2][0] = LIT(0.5) * dcov[2]; dS.m[2][1] = LIT(0.5) * dcov[4]; dS.m[2][2] = dcov[5];
    m3 M2;
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++) M2.m[c][k] = LIT(2.0) * M.m[c][k];
    m3 dM = m3_mul(&M2, &dS);
    m3 Rt = m3_t(&R), dMt = m3_t(&dM);
    for (int c = 0; c < 3; c++)
        dscale[c] = Rt.m[c][0] * dMt.m[c][0] + Rt.m[c][1] * dMt.m[c][1] + Rt.m[c][2] * dMt.m[c][2];
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 3; k++) dMt.m[c][k] *= s[c];
    drot[0] = 2 * z * (dMt.m[0][1] - dMt.m[1][0]) + 2 * y * (dMt.m[2][0] - dMt.m[0][2]) + 2 * x * (dMt.m[1][2] - dMt.m[2][1]);
    drot[1] = 2 * y * (dMt.m[1][0] + dMt.m[0][1]) + 2 * z * (dMt.m[2][0] + dMt.m[0][2]) + 2 * r * (dMt.m[1][2] - dMt.m[2][1]) - 4 * x * (dMt.m[2][2] + dMt.m[1][1]);
    drot[2] = 2 * x * (dMt.m[1][0] + dMt.m[0][1]) + 2 * r * (dMt.m[2][0] - dMt.m[0][2]) + 2 * z * (dMt.m[1][2] + dMt.m[2][1]) - 4 * y * (dMt.m[2][2] + dMt.m[0][0]);
    drot[3] = 2 * r * (dMt.m[0][1] - dMt.m[1][0]) + 2 * x * (dMt.m[2][0] + dMt.m[0][2]) + 2 * y * (dMt.m[1][2] + dMt.m[2][1]) - 4 * z * (dMt.m[1][1] + dMt.m[0][0]);
}

typedef struct {
    int P, D, M, W, H;
    const real *means, *scales, *rots, *shs, *cov3D; /* cov3D: the covariance the forward used */
    const real *view, *proj, *campos;
    real scale_mod, tanx, tany;
    int use_filter, consistent;
    const int *radii;
    const uint8_t *clamped;
    const real *opac; /* consistent mode: mask opacity below the 1e-6 floor */
} SFX(orc_bwd_args);

/* backward.cu:144-274 (computeCov2DCUDA) + :346-396 (preprocessCUDA).
 * dmean2D/dconic/dcolor/dopac come from orc_render_bwd. Outputs dmean3D,
 * dcov3D, dsh, dscale, drot are dense and written for every row. */
void SFX(orc_preprocess_bwd)(const SFX(orc_bwd_args) * a, const real *dmean2D, const real *dconic,
                             const real *dcolor, real *dopac, real *dmean3D, real *dcov3D, real *dsh,
                             real *dscale, real *drot)
{
    const real fy = a->H / (LIT(2.0) * a->tany), fx = a->W / (LIT(2.0) * a->tanx);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < a->P; i++) {
        real *dm = dmean3D + 3 * (size_t)i;
        dm[0] = dm[1] = dm[2] = 0;
        for (int k = 0; k < 6; k++) dcov3D[6 * (size_t)i + k] = 0;
        if (a->M > 0 && dsh) for (int k = 0; k < a->M * 3; k++) dsh[(size_t)i * a->M * 3 + k] = 0;
        if (a->scales) {
            dscale[3 * (size_t)i] = dscale[3 * (size_t)i + 1] = dscale[3 * (size_t)i + 2] = 0;
            drot[4 * (size_t)i] = drot[4 * (size_t)i + 1] = drot[4 * (size_t)i + 2] = drot[4 * (size_t)i + 3] = 0;
        }
        if (!(a->radii[i] > 0)) continue;
        const real *mean = a->means + 3 * (size_t)i;
        const real *cov3D = a->cov3D + 6 * (size_t)i;
        real dcn[3] = {dconic[4 * (size_t)i], dconic[4 * (size_t)i + 1], dconic[4 * (size_t)i + 3]};
        ewa_t e;
        real c00, c01, c11;
        ewa(mean, fx, fy, a->tanx, a->tany, cov3D, a->view, &e, &c00, &c01, &c11);
        real mask_a = 1, mask_c = 1;
        real A, B = c01, C;
        if (a->consistent) {
            if (a->use_filter) {
                if (!((double)c00 > 0.3)) mask_a = 0;
                if (!((double)c11 > 0.3)) mask_c = 0;
                A = dil_max(c00); C = dil_max(c11);
            } else { A = c00; C = c11; }
        } else { A = dil_add(c00); C = dil_add(c11); }
        real denom = A * C - B * B;
        real dL_da = 0, dL_db = 0, dL_dc = 0;
        real d2inv = a->consistent ? LIT(1.0) / (denom * denom) : LIT(1.0) / ((denom * denom) + LIT(0.0000001));
        const m3 *T = &e.T;
        real *dc = dcov3D + 6 * (size_t)i;
        if (d2inv != 0) {
            dL_da = d2inv * (-C * C * dcn[0] + 2 * B * C * dcn[1] + (denom - A * C) * dcn[2]);
            dL_dc = d2inv * (-A * A * dcn[2] + 2 * A * B * dcn[1] + (denom - A * C) * dcn[0]);
            dL_db = d2inv * 2 * (B * C * dcn[0] - (denom + 2 * B * B) * dcn[1] + A * B * dcn[2]);
            dL_da *= mask_a; dL_dc *= mask_c;
            dc[0] = (T->m[0][0] * T->m[0][0] * dL_da + T->m[0][0] * T->m[1][0] * dL_db + T->m[1][0] * T->m[1][0] * dL_dc);
            dc[3] = (T->m[0][1] * T->m[0][1] * dL_da + T->m[0][1] * T->m[1][1] * dL_db + T->m[1][1] * T->m[1][1] * dL_dc);
            dc[5] = (T->m[0][2] * T->m[0][2] * dL_da + T->m[0][2] * T->m[1][2] * dL_db + T->m[1][2] * T->m[1][2] * dL_dc);
            dc[1] = 2 * T->m[0][0] * T->m[0][1] * dL_da + (T->m[0][0] * T->m[1][1] + T->m[0][1] * T->m[1][0]) * dL_db + 2 * T->m[1][0] * T->m[1][1] * dL_dc;
            dc[2] = 2 * T->m[0][0] * T->m[0][2] * dL_da + (T->m[0][0] * T->m[1][2] + T->m[0][2] * T->m[1][0]) * dL_db + 2 * T->m[1][0] * T->m[1][2] * dL_dc;
            dc[4] = 2 * T->m[0][2] * T->m[0][1] * dL_da + (T->m[0][1] * T->m[1][2] + T->m[0][2] * T->m[1][1]) * dL_db + 2 * T->m[1][1] * T->m[1][2] * dL_dc;
        }
        real V[3][3] = {{cov3D[0], cov3D[1], cov3D[2]}, {cov3D[1], cov3D[3], cov3D[4]}, {cov3D[2], cov3D[4], cov3D[5]}};
#define Tm(c, r) (T->m[c][r])
        real dT00 = 2 * (Tm(0, 0) * V[0][0] + Tm(0, 1) * V[0][1] + Tm(0, 2) * V[0][2]) * dL_da + (Tm(1, 0) * V[0][0] + Tm(1, 1) * V[0][1] + Tm(1, 2) * V[0][2]) * dL_db;
        real dT01 = 2 * (Tm(0, 0) * V[1][0] + Tm(0, 1) * V[1][1] + Tm(0, 2) * V[1][2]) * dL_da + (Tm(1, 0) * V[1][0] + Tm(1, 1) * V[1][1] + Tm(1, 2) * V[1][2]) * dL_db;
        real dT02 = 2 * (Tm(0, 0) * V[2][0] + Tm(0, 1) * V[2][1] + Tm(0, 2) * V[2][2]) * dL_da + (Tm(1, 0) * V[2][0] + Tm(1, 1) * V[2][1] + Tm(1, 2) * V[2][2]) * dL_db;
        real dT10 = 2 * (Tm(1, 0) * V[0][0] + Tm(1, 1) * V[0][1] + Tm(1, 2) * V[0][2]) * dL_dc + (Tm(0, 0) * V[0][0] + Tm(0, 1) * V[0][1] + Tm(0, 2) * V[0][2]) * dL_db;
        real dT11 = 2 * (Tm(1, 0) * V[1][0] + Tm(1, 1) * V[1][1] + Tm(1, 2) * V[1][2]) * dL_dc + (Tm(0, 0) * V[1][0] + Tm(0, 1) * V[1][1] + Tm(0, 2) * V[1][2]) * dL_db;
        real dT12 = 2 * (Tm(1, 0) * V[2][0] + Tm(1, 1) * V[2][1] + Tm(1, 2) * V[2][2]) * dL_dc + (Tm(0, 0) * V[2][0] + Tm(0, 1) * V[2][1] + Tm(0, 2) * V[2][2]) * dL_db;
#undef Tm
        const m3 *Wm = &e.W;
        real dJ00 = Wm->m[0][0] * dT00 + Wm->m[0][1] * dT01 + Wm->m[0][2] * dT02;
        real dJ02 = Wm->m[2][0] * dT00 + Wm->m[2][1] * dT01 + Wm->m[2][2] * dT02;
        real dJ11 = Wm->m[1][0] * dT10 + Wm->m[1][1] * dT11 + Wm->m[1][2] * dT12;
        real dJ12 = Wm->m[2][0] * dT10 + Wm->m[2][1] * dT11 + Wm->m[2][2] * dT12;
        real tz = LIT(1.0) / e.t[2], tz2 = tz * tz, tz3 = tz2 * tz;
        real xg = e.xclamp ? 0 : 1, yg = e.yclamp ? 0 : 1;
        real dtx = xg * -fx * tz2 * dJ02;
        real dty = yg * -fy * tz2 * dJ12;
        real dtz = -fx * tz2 * dJ00 - fy * tz2 * dJ11 + (2 * fx * e.t[0]) * tz3 * dJ02 + (2 * fy * e.t[1]) * tz3 * dJ12;
        if (a->consistent) {
            /* a clamped t.x = +-limx * t.z still depends on t.z */
            if (e.xclamp) dtz += (-fx * tz2 * dJ02) * (e.txtz < 0 ? -LIT(1.3) * a->tanx : LIT(1.3) * a->tanx);
            if (e.yclamp) dtz += (-fy * tz2 * dJ12) * (e.tytz < 0 ? -LIT(1.3) * a->tany : LIT(1.3) * a->tany);
        }
        const real *v = a->view;
        dm[0] = v[0] * dtx + v[1] * dty + v[2] * dtz;
        dm[1] = v[4] * dtx + v[5] * dty + v[6] * dtz;
        dm[2] = v[8] * dtx + v[9] * dty + v[10] * dtz;
        /* backward.cu:370-387: screen-space mean gradient through the projection */
        const real *pr = a->proj;
        real mh[4];
        xform4x4(mean, pr, mh);
        real mw = LIT(1.0) / (mh[3] + LIT(0.0000001));
        real mul1 = (pr[0] * mean[0] + pr[4] * mean[1] + pr[8] * mean[2] + pr[12]) * mw * mw;
        real mul2 = (pr[1] * mean[0] + pr[5] * mean[1] + pr[9] * mean[2] + pr[13]) * mw * mw;
        const real *g2 = dmean2D + 3 * (size_t)i;
        dm[0] += (pr[0] * mw - pr[3] * mul1) * g2[0] + (pr[1] * mw - pr[3] * mul2) * g2[1];
        dm[1] += (pr[4] * mw - pr[7] * mul1) * g2[0] + (pr[5] * mw - pr[7] * mul2) * g2[1];
        dm[2] += (pr[8] * mw - pr[11] * mul1) * g2[0] + (pr[9] * mw - pr[11] * mul2) * g2[1];
        if (a->shs && dsh) sh_bwd(i, a->D, a->M, mean, a->campos, a->shs, a->clamped, dcolor, dm, dsh);
        if (a->scales) cov3d_bwd(a->scales + 3 * (size_t)i, a->scale_mod, a->rots + 4 * (size_t)i, dc,
                                 dscale + 3 * (size_t)i, drot + 4 * (size_t)i);
        if (a->consistent && dopac && a->opac && a->opac[i] < LIT(1e-6)) dopac[i] = 0;
    }
}

/* ---------------------------------------------------------------- KPC / GTC statistics */

/* rasterizer_impl.cu:490-556.  out[0]=bar_g_tile, out[1]=used_kv, out[2]=unused_kv,
 * out[3..13]=kpc histogram (11 bins), tile_ratio/tile_total [num_tiles]. */
void SFX(orc_kpc_stats)(long long K, int num_tiles, const real *kv_sum, const uint32_t *kv_cnt,
                        const uint32_t *ranges, float used_thresh, double *out, double *tile_ratio,
                        double *tile_total)
{
    static const float edges[11] = {0.01f, 0.05f, 0.10f, 0.15f, 0.20f, 0.25f, 0.30f, 0.35f, 0.40f, 0.45f, 0.50f};
    unsigned long long bins[11] = {0}, used = 0, unused = 0;
    for (long long k = 0; k < K; k++) {
        if (kv_cnt[k] == 0) { unused++; continue; }
        float v = (float)kv_sum[k];
        int b = 0;
        while (b < 11 && v > edges[b]) b++;
        if (b >= 11) { if (v > edges[10]) continue; b = 10; }
        bins[b]++; used++;
    }
    double gtc = 0;
    for (int t = 0; t < num_tiles; t++) {
        tile_ratio[t] = 0; tile_total[t] = 0;
        uint32_t s = ranges[2 * t], e = ranges[2 * t + 1];
        if (e <= s) continue;
        double sum = 0; uint32_t u = 0;
        tile_total[t] = (double)(e - s);
        for (uint32_t k = s; k < e; k++) {
            sum += (double)(float)kv_sum[k];
            if (kv_cnt[k] > 0 && (float)kv_sum[k] >= used_thresh) u++;
        }
        gtc += sum / (double)(e - s);
        tile_ratio[t] = (double)u / (double)(e - s);
    }
    out[0] = num_tiles > 0 ? gtc / num_tiles : 0;
    out[1] = (double)used; out[2] = (double)unused;
    for (int b = 0; b < 11; b++) out[3 + b] = (double)bins[b];
}

/* ---------------------------------------------------------------- LoD: FilterGS rule */

/* compute_radius_kernel_v2.cu:109-169.  Returns visibility; radius/depth out. */
static int vis_radius_point(int idx, const real *means, const real *lscales, const real *rots, const real *proj,
                            const real *view, real fx, real fy, real tanx, real tany, real pad, real *depth,
                            real *radius)
{
    const real *p = means + 3 * (size_t)idx;
    real ph[4];
    xform4x4(p, proj, ph);
    real pw = LIT(1.0) / (ph[3] + LIT(0.0000001));
    real pp[3] = {ph[0] * pw, ph[1] * pw, ph[2] * pw};
    *depth = pp[2];
    int vis = (pp[2] > LIT(0.0)) && (pp[2] < LIT(1.0)) && (pp[0] > LIT(-1.0) - pad) && (pp[0] < LIT(1.0) + pad) &&
              (pp[1] > LIT(-1.0) - pad) && (pp[1] < LIT(1.0) + pad);
    if (!vis) { *radius = 0; return 0; }
    const real *ls = lscales + 3 * (size_t)idx;
    real s[3] = {EXPR(ls[0]), EXPR(ls[1]), EXPR(ls[2])};
    const real *q0 = rots + 4 * (size_t)idx;
    real nrm = SQRTR(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
    real q[4];
    if (nrm > LIT(0.0)) { q[0] = q0[0] / nrm; q[1] = q0[1] / nrm; q[2] = q0[2] / nrm; q[3] = q0[3] / nrm; }
    else { q[0] = 1; q[1] = q[2] = q[3] = 0; }
    real cov[6];
    cov3d_from(s, LIT(1.0), q, cov);
    ewa_t e;
    real c00, c01, c11;
    ewa(p, fx, fy, tanx, tany, cov, view, &e, &c00, &c01, &c11);
    c00 = dil_max(c00); c11 = dil_max(c11);
    real det = c00 * c11 - c01 * c01;
    if (det <= LIT(0.0)) { *radius = 0; return 1; }
    real mid = LIT(0.5) * (c00 + c11);
    real root = SQRTR(FMAXR(LIT(0.1), mid * mid - det));
    real l1 = mid + root, l2 = mid - root;
    *radius = LIT(3.0) * SQRTR(FMAXR(l1, l2));
    return 1;
}

/* compute_radius_kernel_v2.cu:231-353, with the lazily computed ancestor
 * radius sequentialised (each node's radius is a pure function of the node,
 * so the result does not depend on evaluation order). */
void SFX(orc_visibility_radius)(int P, const real *means, const real *lscales, const real *rots, const real *proj,
                                const real *view, const int32_t *node_index, const int32_t *anc, int L, real fx,
                                real fy, real tanx, real tany, real pad, real rmax, real rfilt, uint8_t *mask,
                                real *radius2d, real *depth)
{
    uint8_t *vis = malloc(P > 0 ? P : 1);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P; i++)
        vis[i] = (uint8_t)vis_radius_point(i, means, lscales, rots, proj, view, fx, fy, tanx, tany, pad, &depth[i],
                                           &radius2d[i]);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P; i++) {
        if (!vis[i]) { mask[i] = 0; continue; }
        int keep = 1;
        if (node_index[i] != -1) keep = radius2d[i] <= rmax;
        else {
            for (int l = 0; l < L; l++) {
                int32_t a = anc[(size_t)i * L + l];
                if (a < 0) break;
                if (a == i) continue;
                if (node_index[a] == -1) continue;
                real ar = radius2d[a];
                if (ar > LIT(0.0) && ar <= rmax) { keep = 0; break; }
            }
        }
        if (keep && rfilt > LIT(0.0) && radius2d[i] > rfilt) keep = 0;
        mask[i] = (uint8_t)keep;
    }
    free(vis);
}

/* ---------------------------------------------------------------- LoD: LoG cut rule */

/* LoG/model/tensor_tree.py:133-187 (TensorTree.traverse) with radius from the
 * v2 3-sigma kernel on activated parameters (LoG/model/level_of_gaussian.py:66-88),
 * given here as a precomputed per-node radius array.  Output: node ids in
 * traversal order (roots kept, then each level's kept children in frontier
 * order).  Returns the count.  tree: [num_tree_nodes, max_child], -1 = none. */
long long SFX(orc_log_cut)(int num_roots, const int32_t *roots, const int32_t *node_index, const int32_t *tree,
                           int max_child, const real *radius, real min_res, int max_depth, int32_t *out,
                           int32_t *scratch_a, int32_t *scratch_b)
{
    long long n = 0, nf = 0;
    for (int r = 0; r < num_roots; r++) {
        int32_t id = roots[r];
        if (radius[id] < min_res || node_index[id] == -1) out[n++] = id;
        else scratch_a[nf++] = id;
    }
    int32_t *front = scratch_a, *next = scratch_b;
    int level = 1;
    while (1) {
        if (level > 30 || level > max_depth) {
            for (long long k = 0; k < nf; k++) out[n++] = front[k];
            break;
        }
        long long nn = 0;
        /* children listed frontier-major, child-slot-minor; kept ones are
         * appended in that order, then the expanded ones become the frontier */
        for (long long k = 0; k < nf; k++) {
            int32_t ni = node_index[front[k]];
            for (int c = 0; c < max_child; c++) {
                int32_t ch = tree[(size_t)ni * max_child + c];
                if (ch == -1) continue;
                if (radius[ch] < min_res || node_index[ch] == -1) out[n++] = ch;
            }
        }
        for (long long k = 0; k < nf; k++) {
            int32_t ni = node_index[front[k]];
            for (int c = 0; c < max_child; c++) {
                int32_t ch = tree[(size_t)ni * max_child + c];
                if (ch == -1) continue;
                if (!(radius[ch] < min_res || node_index[ch] == -1)) next[nn++] = ch;
            }
        }
        if (nn == 0) break;
        int32_t *t = front; front = next; next = t;
        nf = nn;
        level++;
    }
    return n;
}

/* ---------------------------------------------------------------- ancestor_path */

/* apps/ancestor.py:21-73 (rebuild_ancestor_path), level by level as written:
 * for level = 1 .. max(depth), the nodes at that level with a parent p >= 0
 * take a copy of row(p) as it stands before this level's writes, then column
 * level-1 = p; nodes with p < 0 keep -1.  The gather of a level is finished
 * before its scatter (torch evaluates the right-hand side first), so a node
 * whose parent sits in the same level copies the parent's old row.  Returns 0,
 * or -1 where the reference raises an index error (parent id >= P, or column
 * level-1 >= L for a node with a parent).  out: [P, L], scratch: [P * L]. */
int SFX(orc_ancestor_path)(int P, const int32_t *parent, const int32_t *depth, int L, int32_t *out,
                           int32_t *scratch)
{
    for (size_t k = 0; k < (size_t)P * (size_t)L; k++) out[k] = -1;
    if (P == 0 || L == 0) return 0;
    int max_depth = 0;
    for (int i = 0; i < P; i++)
        if (depth[i] > max_depth) max_depth = depth[i];
    for (int level = 1; level <= max_depth; level++) {
        /* gather: rows of the parents as they are now */
        for (int i = 0; i < P; i++) {
            if (depth[i] != level || parent[i] < 0) continue;
            if (parent[i] >= P) return -1;
            memcpy(scratch + (size_t)i * L, out + (size_t)parent[i] * L, sizeof(int32_t) * (size_t)L);
        }
        /* scatter */
        for (int i = 0; i < P; i++) {
            if (depth[i] != level) continue;
            if (parent[i] < 0) {
                for (int k = 0; k < L; k++) out[(size_t)i * L + k] = -1;
                continue;
            }
            if (level - 1 >= L) return -1;
            memcpy(out + (size_t)i * L, scratch + (size_t)i * L, sizeof(int32_t) * (size_t)L);
            out[(size_t)i * L + level - 1] = parent[i];
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- activations + gather */

/* LoG/model/activation.py:36-43 + sh_utils.py:31-74, applied to gathered rows
 * (FilterGS/filtergs.py:98-134): exp scale, sigmoid opacity, normalised quat
 * (torch F.normalize: q / max(|q|, 1e-12)), colour = SH2RGB(dc) + eval_sh_wobase. */
void SFX(orc_gather_activate)(long long N, const int64_t *index, const real *xyz, const real *lscale, const real *rot,
                              const real *opac, const real *dc, const real *shs_rest, int sh_deg, int rest_coeffs,
                              const real *campos, real *o_xyz, real *o_scale, real *o_rot, real *o_opac, real *o_rgb)
{
    const real C0 = (real)SH_C0, C1 = (real)SH_C1;
#pragma omp parallel for schedule(static)
    for (long long n = 0; n < N; n++) {
        int64_t s = index[n];
        for (int k = 0; k < 3; k++) o_xyz[3 * n + k] = xyz[3 * s + k];
        for (int k = 0; k < 3; k++) o_scale[3 * n + k] = EXPR(lscale[3 * s + k]);
        const real *q = rot + 4 * s;
        real nr = SQRTR(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (nr < LIT(1e-12)) nr = LIT(1e-12);
        for (int k = 0; k < 4; k++) o_rot[4 * n + k] = q[k] / nr;
        o_opac[n] = LIT(1.0) / (LIT(1.0) + EXPR(-opac[s]));
        real d[3] = {xyz[3 * s] - campos[0], xyz[3 * s + 1] - campos[1], xyz[3 * s + 2] - campos[2]};
        real dl = SQRTR(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        real x = d[0] / dl, y = d[1] / dl, z = d[2] / dl;
        for (int c = 0; c < 3; c++) {
            real col = dc[3 * s + c] * C0 + LIT(0.5);
            if (sh_deg > 0 && shs_rest) {
                const real *sh = shs_rest + (size_t)s * rest_coeffs * 3;
#define R(k) sh[(k) * 3 + c]
                real r = -C1 * y * R(0) + C1 * z * R(1) - C1 * x * R(2);
                if (sh_deg > 1) {
                    real xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
                    r = r + (real)SH_C2[0] * xy * R(3) + (real)SH_C2[1] * yz * R(4) +
                        (real)SH_C2[2] * (2 * zz - xx - yy) * R(5) + (real)SH_C2[3] * xz * R(6) + (real)SH_C2[4] * (xx - yy) * R(7);
                    if (sh_deg > 2)
                        r = r + (real)SH_C3[0] * y * (3 * xx - yy) * R(8) + (real)SH_C3[1] * xy * z * R(9) +
                            (real)SH_C3[2] * y * (4 * zz - xx - yy) * R(10) + (real)SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * R(11) +
                            (real)SH_C3[4] * x * (4 * zz - xx - yy) * R(12) + (real)SH_C3[5] * z * (xx - yy) * R(13) +
                            (real)SH_C3[6] * x * (xx - 3 * yy) * R(14);
                }
#undef R
                col += r;
            }
            o_rgb[3 * n + c] = col;
        }
    }
}

int SFX(orc_num_threads)(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void SFX(orc_set_threads)(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
