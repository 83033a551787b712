"""The reference build's FP32 arithmetic for the per-Gaussian preprocess, bit for bit, in numpy.

TEST INFRASTRUCTURE ONLY: the tests use it to build inputs the reference must see bit for
bit (a precomputed covariance equal to the one the CUDA path computes) and to pin, on the
CPU, the multiply-add grouping that the CUDA kernels write out.

nvcc fuses a product into the following add or subtract wherever it can (a fused
multiply-add rounds once).  Which product of a sum gets fused depends on how the compiler
sees the expression, so the reference build's choices were found by comparing candidate
groupings with its outputs (every visible Gaussian of three 1080p views of the 2M-Gaussian
urban scene, and the golden fixtures under tests/golden).  This module evaluates:

  cov3d     computeCov3D (antialias/cuda_rasterizer/forward.cu:151-185)
  view_z    transformPoint4x3(...).z (auxiliary.h:58-66)
  conic     computeCov2D (forward.cu:102-146), the dilation, det and inverse (forward.cu:326-332)
  sh_rgb    computeColorFromSH (forward.cu:48-99)

Every product and quotient is a correctly rounded FP32 operation (numpy float32), every
fused multiply-add is computed exactly and rounded once (`fma`).
"""
import numpy as np

f32, f64 = np.float32, np.float64

C0 = f32(0.28209479177387814)
C1 = f32(0.4886025119029199)
C2 = [f32(v) for v in (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792,
                       0.5462742152960396)]
C3 = [f32(v) for v in (-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
                       -0.4570457994644658, 1.445305721320277, -0.5900435899266435)]


def _a(x):
    return np.asarray(x, f32)


def fma(a, b, c):
    """a*b + c rounded once to FP32.  The FP64 product of two FP32 values is exact; the FP64 sum
    t may round, and rounding t again to FP32 is wrong only when t lands exactly halfway
    between two FP32 values -- those ties are broken by the sign of the FP64 sum's error."""
    a, b, c = np.broadcast_arrays(_a(a).astype(f64), _a(b).astype(f64), _a(c).astype(f64))
    p = a * b
    t = p + c
    e = (p - (t - (t - p))) + (c - (t - p))          # TwoSum: p + c == t + e exactly
    r = t.astype(f32)
    rb = r.astype(f64)
    with np.errstate(invalid="ignore", over="ignore"):
        other = np.nextafter(r, np.where(t > rb, f32(np.inf), f32(-np.inf))).astype(f64)
        tie = (t != rb) & (2.0 * t == rb + other) & (e != 0)
    if np.any(tie):
        hi, lo = np.maximum(rb, other), np.minimum(rb, other)
        r = np.where(tie, np.where(e > 0, hi, lo).astype(f32), r)
    return np.asarray(r, f32)


def mul(a, b):
    return (_a(a) * _a(b)).astype(f32)


def add(a, b):
    return (_a(a) + _a(b)).astype(f32)


def sub(a, b):
    return (_a(a) - _a(b)).astype(f32)


def div(a, b):
    with np.errstate(divide="ignore", invalid="ignore"):
        return (_a(a) / _a(b)).astype(f32)


def dot3(a0, b0, a1, b1, a2, b2):
    """((a0 b0 + a1 b1) + a2 b2) with the first and the last product fused."""
    return fma(a2, b2, fma(a0, b0, mul(a1, b1)))


def cov3d(scales, rots, mod=1.0):
    """[P,6] upper triangle of Sigma = (S R)^T (S R), rotations (r, x, y, z) used as given."""
    q = _a(rots)
    r, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    one, two = f32(1), f32(2)
    R = [[None] * 3 for _ in range(3)]                 # R[c][k]: glm column c, row k
    R[0][0] = sub(one, mul(two, add(mul(y, y), mul(z, z))))   # y y and z z left unfused
    R[0][1] = mul(two, fma(x, y, -mul(r, z)))
    R[0][2] = mul(two, fma(r, y, mul(x, z)))                  # x z (shared with R[2][0]) unfused
    R[1][0] = mul(two, fma(x, y, mul(r, z)))
    R[1][1] = sub(one, mul(two, fma(x, x, mul(z, z))))
    R[1][2] = mul(two, fma(y, z, -mul(r, x)))
    R[2][0] = mul(two, fma(-r, y, mul(x, z)))
    R[2][1] = mul(two, fma(y, z, mul(r, x)))
    R[2][2] = sub(one, mul(two, fma(x, x, mul(y, y))))
    s = mul(f32(mod), _a(scales))
    M = [[mul(s[:, k], R[c][k]) for k in range(3)] for c in range(3)]

    def sig(c, k):
        return dot3(M[k][0], M[c][0], M[k][1], M[c][1], M[k][2], M[c][2])

    return np.stack([sig(0, 0), sig(0, 1), sig(0, 2), sig(1, 1), sig(1, 2), sig(2, 2)], 1)


def _xform(v, p, r):
    return add(dot3(v[r], p[:, 0], v[4 + r], p[:, 1], v[8 + r], p[:, 2]), v[12 + r])


def view_z(means, viewmatrix):
    """The view-space depth transformPoint4x3(mean, viewmatrix).z."""
    return _xform(_a(viewmatrix).reshape(-1), _a(means), 2)


def conic(means, cov3D, viewmatrix, W, H, tanfovx, tanfovy, use_filter=True):
    """[P,3] inverse 2D covariance (conic.x, conic.y, conic.z) and [P] det, from a [P,6] cov3D."""
    v = _a(viewmatrix).reshape(-1)
    m = _a(means)
    tanx, tany = f32(tanfovx), f32(tanfovy)
    fx, fy = div(f32(W), mul(f32(2), tanx)), div(f32(H), mul(f32(2), tany))
    tx, ty, tz = _xform(v, m, 0), _xform(v, m, 1), _xform(v, m, 2)
    limx, limy = mul(f32(1.3), tanx), mul(f32(1.3), tany)
    tx = mul(np.minimum(limx, np.maximum(-limx, div(tx, tz))), tz)
    ty = mul(np.minimum(limy, np.maximum(-limy, div(ty, tz))), tz)
    tz2 = mul(tz, tz)
    j00, j02 = div(fx, tz), div(-mul(fx, tx), tz2)
    j11, j12 = div(fy, tz), div(-mul(fy, ty), tz2)
    T = [[fma(v[4 * k + 2], j02, mul(v[4 * k], j00)) for k in range(3)],
         [fma(v[4 * k + 2], j12, mul(v[4 * k + 1], j11)) for k in range(3)]]
    c = _a(cov3D)
    V = [[c[:, 0], c[:, 1], c[:, 2]], [c[:, 1], c[:, 3], c[:, 4]], [c[:, 2], c[:, 4], c[:, 5]]]
    X = [[dot3(T[k][0], V[0][j], T[k][1], V[1][j], T[k][2], V[2][j]) for k in range(2)] for j in range(3)]

    def cv(j, k):
        return dot3(X[0][k], T[j][0], X[1][k], T[j][1], X[2][k], T[j][2])

    a, b, cc = cv(0, 0), cv(0, 1), cv(1, 1)
    if use_filter:                                      # DILATE_PIXEL is a double literal
        a = np.maximum(a.astype(f64), 0.3).astype(f32)
        cc = np.maximum(cc.astype(f64), 0.3).astype(f32)
    det = fma(a, cc, -mul(b, b))
    inv = div(f32(1), det)
    return np.stack([mul(cc, inv), mul(-b, inv), mul(a, inv)], 1), det


def sh_rgb(means, campos, shs, degree):
    """[P,3] clamped colour and [P,3] clamp flags of SH degree <= 3 rows shs [P,M,3]."""
    d = sub(_a(means), _a(campos)[None])
    ln = np.sqrt(dot3(d[:, 0], d[:, 0], d[:, 1], d[:, 1], d[:, 2], d[:, 2]).astype(f64)).astype(f32)
    x, y, z = (div(d[:, i], ln)[:, None] for i in range(3))
    s = [_a(shs)[:, k, :] for k in range(_a(shs).shape[1])]
    r = mul(C0, s[0])
    if degree > 0:
        r = fma(-mul(C1, y), s[1], r)
        r = fma(mul(C1, z), s[2], r)
        r = fma(-mul(C1, x), s[3], r)
        if degree > 1:
            xx, yy, zz = mul(x, x), mul(y, y), mul(z, z)
            xy, yz, xz = mul(x, y), mul(y, z), mul(x, z)
            f = [mul(C2[0], xy), mul(C2[1], yz), mul(C2[2], sub(sub(mul(f32(2), zz), xx), yy)), mul(C2[3], xz),
                 mul(C2[4], sub(xx, yy))]
            for i in range(5):
                r = fma(f[i], s[4 + i], r)
            if degree > 2:
                q4 = sub(sub(mul(f32(4), zz), xx), yy)
                g = [mul(mul(C3[0], y), fma(f32(3), xx, -yy)), mul(mul(C3[1], xy), z), mul(mul(C3[2], y), q4),
                     mul(mul(C3[3], z), fma(f32(-3), yy, fma(f32(-3), xx, mul(f32(2), zz)))),
                     mul(mul(C3[4], x), q4), mul(mul(C3[5], z), sub(xx, yy)),
                     mul(mul(C3[6], x), fma(f32(-3), yy, xx))]
                for i in range(7):
                    r = fma(g[i], s[9 + i], r)
    r = add(r, f32(0.5))
    return np.maximum(r, f32(0)), r < 0
