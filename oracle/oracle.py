"""Python (ctypes + numpy) front end of the C oracle in fgs_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, always as the checker, never as the product.

Every function mirrors a reference routine (cited in fgs_oracle.c) and works on
numpy arrays in the reference's layouts: means [P,3], scales [P,3], rotations
[P,4] (w,x,y,z), opacities [P], shs [P,M,3], column-major (transposed) 4x4
view/projection matrices as 16 floats.  `dtype` picks the FP32 restatement
(np.float32) or the FP64 evaluation of the same equations (np.float64).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "fgs_oracle.c")
BUILD = os.path.join(HERE, "build")
LIBS = {np.float32: os.path.join(BUILD, "libfgs_oracle_f32.so"),
        np.float64: os.path.join(BUILD, "libfgs_oracle_f64.so")}


def build(force=False):
    """Compile the oracle twice (float / double).  Plain gcc, no FMA contraction."""
    os.makedirs(BUILD, exist_ok=True)
    for dt, out in LIBS.items():
        if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
            continue
        extra = ["-DREAL=double", "-DORC_F64"] if dt is np.float64 else []
        cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
               "-o", out, SRC, "-lm"] + extra
        subprocess.check_call(cmd)


def build_tile_variant(block_x, block_y, out_dir):
    """FP32 oracle binning into block_x x block_y tiles, lambda_G's exponent kept at the reference's 256
    (the tile-shape study; the reference itself bins into 16 x 16).  Returns the loaded library, to be
    passed as `lib=` with `tile=(block_x, block_y)` to bin_pairs and as `lib=` to preprocess and render."""
    out = os.path.join(out_dir, f"libfgs_oracle_f32_{block_x}x{block_y}.so")
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
                           "-o", out, SRC, "-lm", f"-DBLOCK_X={int(block_x)}", f"-DBLOCK_Y={int(block_y)}",
                           "-DOGFS_LAMBDA_PIXELS=256"])
    return C.CDLL(out)


_libs = {}


def _lib(dtype):
    dt = np.dtype(dtype).type
    if dt not in _libs:
        if not os.path.exists(LIBS[dt]) or os.path.getmtime(LIBS[dt]) < os.path.getmtime(SRC):
            build()
        _libs[dt] = C.CDLL(LIBS[dt])
    return _libs[dt]


def _sfx(dtype):
    return "_f64" if np.dtype(dtype) == np.float64 else "_f32"


def _real(dtype):
    return C.c_double if np.dtype(dtype) == np.float64 else C.c_float


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _arr(x, dtype):
    if x is None:
        return None
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


def set_threads(n):
    for dt in (np.float32, np.float64):
        getattr(_lib(dt), "orc_set_threads" + _sfx(dt))(int(n))


def num_threads():
    return getattr(_lib(np.float32), "orc_num_threads_f32")()


def _pre_struct(dtype):
    R = _real(dtype)
    return type("PreArgs", (C.Structure,), {"_fields_": [
        ("P", C.c_int), ("D", C.c_int), ("M", C.c_int), ("W", C.c_int), ("H", C.c_int),
        ("means", C.c_void_p), ("scales", C.c_void_p), ("rots", C.c_void_p), ("opac", C.c_void_p),
        ("shs", C.c_void_p), ("cov3D_precomp", C.c_void_p), ("colors_precomp", C.c_void_p),
        ("view", C.c_void_p), ("proj", C.c_void_p), ("campos", C.c_void_p),
        ("scale_mod", R), ("tanx", R), ("tany", R), ("use_filter", C.c_int),
        ("eps_scale", R), ("eps_max", R), ("energy_floor", R), ("ratio_min", R), ("filter3d", R)]})


def _bwd_struct(dtype):
    R = _real(dtype)
    return type("BwdArgs", (C.Structure,), {"_fields_": [
        ("P", C.c_int), ("D", C.c_int), ("M", C.c_int), ("W", C.c_int), ("H", C.c_int),
        ("means", C.c_void_p), ("scales", C.c_void_p), ("rots", C.c_void_p), ("shs", C.c_void_p),
        ("cov3D", C.c_void_p), ("view", C.c_void_p), ("proj", C.c_void_p), ("campos", C.c_void_p),
        ("scale_mod", R), ("tanx", R), ("tany", R), ("use_filter", C.c_int), ("consistent", C.c_int),
        ("radii", C.c_void_p), ("clamped", C.c_void_p), ("opac", C.c_void_p)]})


class Scene:
    """Inputs of one rasterizer call, in the reference's argument meaning."""

    def __init__(self, means3D, opacities, W, H, tanfovx, tanfovy, viewmatrix, projmatrix, campos,
                 bg=(0, 0, 0), shs=None, sh_degree=0, colors_precomp=None, scales=None, rotations=None,
                 cov3D_precomp=None, scale_modifier=1.0, use_filter=True, ogfs=(0.2, 0.2, 0.05, 0.7),
                 filter3d=0.0):
        self.means3D, self.opacities = means3D, opacities
        self.W, self.H, self.tanfovx, self.tanfovy = int(W), int(H), float(tanfovx), float(tanfovy)
        self.viewmatrix, self.projmatrix, self.campos = viewmatrix, projmatrix, campos
        self.bg, self.shs, self.sh_degree, self.colors_precomp = bg, shs, int(sh_degree), colors_precomp
        self.scales, self.rotations, self.cov3D_precomp = scales, rotations, cov3D_precomp
        self.scale_modifier, self.use_filter, self.ogfs, self.filter3d = float(scale_modifier), bool(use_filter), ogfs, float(filter3d)


def preprocess(sc, dtype=np.float32, lib=None):
    lib = lib or _lib(dtype)
    f = getattr(lib, "orc_preprocess" + _sfx(dtype))
    P = int(np.asarray(sc.means3D).shape[0])
    A = {k: _arr(getattr(sc, k), dtype) for k in ("means3D", "scales", "rotations", "opacities", "shs",
                                                    "cov3D_precomp", "colors_precomp", "viewmatrix",
                                                    "projmatrix", "campos")}
    M = 0 if A["shs"] is None else int(A["shs"].shape[1])
    S = _pre_struct(dtype)
    a = S(P, sc.sh_degree, M, sc.W, sc.H, _p(A["means3D"]), _p(A["scales"]), _p(A["rotations"]),
          _p(A["opacities"].reshape(-1)), _p(A["shs"]), _p(A["cov3D_precomp"]), _p(A["colors_precomp"]),
          _p(A["viewmatrix"]), _p(A["projmatrix"]), _p(A["campos"]), sc.scale_modifier, sc.tanfovx, sc.tanfovy,
          int(sc.use_filter), *[float(v) for v in sc.ogfs], sc.filter3d)
    out = dict(radii=np.zeros(P, np.int32), means2D=np.zeros((P, 2), dtype), depths=np.zeros(P, dtype),
               conic_opacity=np.zeros((P, 4), dtype), rgb=np.zeros((P, 3), dtype),
               clamped=np.zeros((P, 3), np.uint8), tiles_touched=np.zeros(P, np.uint32),
               cov3D=np.zeros((P, 6), dtype))
    f(C.byref(a), *[_p(out[k]) for k in ("radii", "means2D", "depths", "conic_opacity", "rgb", "clamped",
                                         "tiles_touched", "cov3D")])
    out["_keep"] = A
    return out


def compute_radius(variant, means, scales, rotations, view, proj, fx, fy, tanx, tany, dtype=np.float32):
    """variant 0: antialias _C.compute_radius; variant 1: FilterGS/LoG v2 compute_radius."""
    lib = _lib(dtype)
    R = _real(dtype)
    means, scales, rotations = _arr(means, dtype), _arr(scales, dtype), _arr(rotations, dtype)
    view, proj = _arr(view, dtype), _arr(proj, dtype)
    P = means.shape[0]
    out = np.zeros(P, dtype)
    getattr(lib, "orc_compute_radius" + _sfx(dtype))(
        C.c_int(variant), C.c_int(P), _p(means), _p(scales), _p(rotations), _p(view), _p(proj),
        R(fx), R(fy), R(tanx), R(tany), _p(out))
    return out


def mark_visible(means, view, dtype=np.float32):
    means, view = _arr(means, dtype), _arr(view, dtype)
    out = np.zeros(means.shape[0], np.uint8)
    getattr(_lib(dtype), "orc_mark_visible" + _sfx(dtype))(C.c_int(means.shape[0]), _p(means), _p(view), _p(out))
    return out.astype(bool)


def bin_pairs(pre, W, H, dtype=np.float32, lib=None, tile=(16, 16)):
    """Duplicate + stable sort + tile ranges: (sorted keys u64, sorted values u32, ranges [T,2] u32).
    `tile` is the binning tile the library was built with (build_tile_variant)."""
    lib = lib or _lib(dtype)
    K = int(pre["tiles_touched"].astype(np.int64).sum())
    gx, gy = (W + tile[0] - 1) // tile[0], (H + tile[1] - 1) // tile[1]
    keys = np.zeros(max(K, 1), np.uint64)
    vals = np.zeros(max(K, 1), np.uint32)
    ranges = np.zeros((gx * gy, 2), np.uint32)
    f = getattr(lib, "orc_bin" + _sfx(dtype))
    f.restype = C.c_longlong
    n = f(C.c_int(len(pre["radii"])), C.c_int(W), C.c_int(H), _p(pre["radii"]), _p(pre["means2D"]),
          _p(pre["depths"]), _p(keys), _p(vals), _p(ranges))
    assert n == K, (n, K)
    return keys[:K], vals[:K], ranges


def render(sc, pre, vals, ranges, dtype=np.float32, stats=False, tile_range=(-1, -1), lib=None):
    lib = lib or _lib(dtype)
    W, H = sc.W, sc.H
    P = len(pre["radii"])
    feat = _arr(sc.colors_precomp, dtype) if sc.colors_precomp is not None else pre["rgb"]
    bg = _arr(sc.bg, dtype)
    K = len(vals)
    out = dict(color=np.zeros((3, H, W), dtype), final_T=np.zeros(H * W, dtype),
               n_contrib=np.zeros(H * W, np.uint32), point_id=np.zeros(H * W, np.int32),
               point_weight_pixel=np.zeros(H * W, dtype), point_weight=np.zeros(P, dtype))
    kv_sum = np.zeros(max(K, 1), dtype) if stats else None
    kv_cnt = np.zeros(max(K, 1), np.uint32) if stats else None
    getattr(lib, "orc_render" + _sfx(dtype))(
        C.c_int(W), C.c_int(H), _p(ranges), _p(vals), _p(pre["means2D"]), _p(feat), _p(pre["conic_opacity"]),
        _p(bg), _p(out["color"]), _p(out["final_T"]), _p(out["n_contrib"]), _p(out["point_id"]),
        _p(out["point_weight_pixel"]), _p(out["point_weight"]), _p(kv_sum), _p(kv_cnt),
        C.c_int(tile_range[0]), C.c_int(tile_range[1]))
    if stats:
        out["kv_sum"], out["kv_cnt"] = kv_sum[:K], kv_cnt[:K]
    return out


def kpc_stats(kv_sum, kv_cnt, ranges, used_thresh=1e-4, dtype=np.float32):
    lib = _lib(dtype)
    T = ranges.shape[0]
    out = np.zeros(14, np.float64)
    tr, tt = np.zeros(T, np.float64), np.zeros(T, np.float64)
    getattr(lib, "orc_kpc_stats" + _sfx(dtype))(
        C.c_longlong(len(kv_sum)), C.c_int(T), _p(_arr(kv_sum, dtype)), _p(np.ascontiguousarray(kv_cnt, np.uint32)),
        _p(np.ascontiguousarray(ranges, np.uint32)), C.c_float(used_thresh), _p(out), _p(tr), _p(tt))
    return dict(bar_g=out[0], used_kv_pairs=out[1], unused_kv_pairs=out[2], kpc_hist=out[3:14],
                tile_ratio=tr, tile_total_kv=tt)


def forward(sc, dtype=np.float32, stats=False):
    """Full forward: preprocess, binning, render.  Returns a dict with every intermediate."""
    pre = preprocess(sc, dtype)
    keys, vals, ranges = bin_pairs(pre, sc.W, sc.H, dtype)
    r = render(sc, pre, vals, ranges, dtype, stats=stats)
    r.update(pre=pre, keys=keys, vals=vals, ranges=ranges, num_rendered=len(vals))
    return r


def backward(sc, fwd, dL_dimage, dtype=np.float32, consistent=False, tile_range=(-1, -1)):
    """Gradients in the reference's return meaning: dict of means2D, colors, opacity, means3D, cov3D,
    sh, scales, rotations (dense, [P,...])."""
    lib = _lib(dtype)
    pre = fwd["pre"]
    P = len(pre["radii"])
    W, H = sc.W, sc.H
    feat = _arr(sc.colors_precomp, dtype) if sc.colors_precomp is not None else pre["rgb"]
    g = dict(means2D=np.zeros((P, 3), dtype), conic=np.zeros((P, 4), dtype), opacity=np.zeros(P, dtype),
             colors=np.zeros((P, 3), dtype))
    dpix = _arr(dL_dimage, dtype)
    getattr(lib, "orc_render_bwd" + _sfx(dtype))(
        C.c_int(W), C.c_int(H), _p(fwd["ranges"]), _p(fwd["vals"]), _p(pre["means2D"]), _p(feat),
        _p(pre["conic_opacity"]), _p(_arr(sc.bg, dtype)), _p(fwd["final_T"]), _p(fwd["n_contrib"]), _p(dpix),
        _p(g["means2D"]), _p(g["conic"]), _p(g["opacity"]), _p(g["colors"]), C.c_int(int(consistent)),
        C.c_int(tile_range[0]), C.c_int(tile_range[1]))
    A = pre["_keep"]
    M = 0 if A["shs"] is None else int(A["shs"].shape[1])
    S = _bwd_struct(dtype)
    cov = A["cov3D_precomp"] if (A["cov3D_precomp"] is not None and sc.filter3d == 0) else pre["cov3D"]
    a = S(P, sc.sh_degree, M, W, H, _p(A["means3D"]), _p(A["scales"]), _p(A["rotations"]), _p(A["shs"]),
          _p(cov), _p(A["viewmatrix"]), _p(A["projmatrix"]), _p(A["campos"]), sc.scale_modifier, sc.tanfovx,
          sc.tanfovy, int(sc.use_filter), int(consistent), _p(pre["radii"]), _p(pre["clamped"]),
          _p(A["opacities"].reshape(-1)))
    out = dict(means3D=np.zeros((P, 3), dtype), cov3D=np.zeros((P, 6), dtype),
               sh=np.zeros((P, M, 3), dtype), scales=np.zeros((P, 3), dtype), rotations=np.zeros((P, 4), dtype))
    getattr(lib, "orc_preprocess_bwd" + _sfx(dtype))(
        C.byref(a), _p(g["means2D"]), _p(g["conic"]), _p(g["colors"]), _p(g["opacity"]), _p(out["means3D"]),
        _p(out["cov3D"]), _p(out["sh"]) if M > 0 else None, _p(out["scales"]), _p(out["rotations"]))
    out.update(means2D=g["means2D"], colors=g["colors"], opacity=g["opacity"].reshape(P, 1), conic=g["conic"])
    return out


def visibility_radius(means, lscales, rots, proj, view, node_index, ancestor_path, fx, fy, tanx, tany,
                      padding, radius_max, radius_filter_threshold, dtype=np.float32):
    lib = _lib(dtype)
    R = _real(dtype)
    means, lscales, rots = _arr(means, dtype), _arr(lscales, dtype), _arr(rots, dtype)
    proj, view = _arr(proj, dtype), _arr(view, dtype)
    ni = np.ascontiguousarray(node_index, np.int32)
    anc = np.ascontiguousarray(ancestor_path, np.int32)
    P, L = means.shape[0], (anc.shape[1] if anc.ndim == 2 else 0)
    mask = np.zeros(P, np.uint8)
    rad, dep = np.zeros(P, dtype), np.zeros(P, dtype)
    getattr(lib, "orc_visibility_radius" + _sfx(dtype))(
        C.c_int(P), _p(means), _p(lscales), _p(rots), _p(proj), _p(view), _p(ni), _p(anc), C.c_int(L),
        R(fx), R(fy), R(tanx), R(tany), R(padding), R(radius_max), R(radius_filter_threshold),
        _p(mask), _p(rad), _p(dep))
    return mask.astype(bool), rad, dep


def log_cut(roots, node_index, tree, radius, min_res, max_depth=1000, dtype=np.float32):
    """LoG TensorTree.traverse order of the selected node ids (int64)."""
    lib = _lib(dtype)
    R = _real(dtype)
    roots = np.ascontiguousarray(roots, np.int32)
    ni = np.ascontiguousarray(node_index, np.int32)
    tree = np.ascontiguousarray(tree, np.int32)
    rad = _arr(radius, dtype)
    P = ni.shape[0]
    out = np.zeros(P + 1, np.int32)
    sa, sb = np.zeros(P + 1, np.int32), np.zeros(P + 1, np.int32)
    f = getattr(lib, "orc_log_cut" + _sfx(dtype))
    f.restype = C.c_longlong
    n = f(C.c_int(len(roots)), _p(roots), _p(ni), _p(tree), C.c_int(tree.shape[1] if tree.ndim == 2 else 1),
          _p(rad), R(min_res), C.c_int(max_depth), _p(out), _p(sa), _p(sb))
    return out[:n].astype(np.int64)


def ancestor_path(parent, depth, L):
    """rebuild_ancestor_path (apps/ancestor.py:21-73) -> int32 [P, L], or None where the reference raises."""
    lib = _lib(np.float32)
    par = np.ascontiguousarray(parent, np.int32)
    dep = np.ascontiguousarray(depth, np.int32)
    P = par.shape[0]
    out = np.zeros((P, L), np.int32)
    scratch = np.zeros((P, L), np.int32)
    f = lib.orc_ancestor_path_f32
    f.restype = C.c_int
    rc = f(C.c_int(P), _p(par), _p(dep), C.c_int(L), _p(out), _p(scratch))
    return None if rc else out


def gather_activate(index, xyz, lscale, rot, opac, dc, shs_rest, sh_deg, campos, dtype=np.float32):
    lib = _lib(dtype)
    index = np.ascontiguousarray(index, np.int64)
    N = index.shape[0]
    xyz, lscale, rot, opac, dc = (_arr(v, dtype) for v in (xyz, lscale, rot, opac, dc))
    rest = _arr(shs_rest, dtype) if shs_rest is not None else None
    rc = 0 if rest is None else int(rest.shape[1])
    o = dict(xyz=np.zeros((N, 3), dtype), scaling=np.zeros((N, 3), dtype), rotation=np.zeros((N, 4), dtype),
             opacity=np.zeros((N, 1), dtype), colors=np.zeros((N, 3), dtype))
    getattr(lib, "orc_gather_activate" + _sfx(dtype))(
        C.c_longlong(N), _p(index), _p(xyz), _p(lscale), _p(rot), _p(opac.reshape(-1)), _p(dc), _p(rest),
        C.c_int(sh_deg), C.c_int(rc), _p(_arr(campos, dtype)), _p(o["xyz"]), _p(o["scaling"]), _p(o["rotation"]),
        _p(o["opacity"]), _p(o["colors"]))
    return o
