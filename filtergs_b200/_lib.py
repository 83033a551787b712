"""ctypes binding of libfiltergs_b200.so (the C ABI declared in include/filtergs_b200.h).

The library is built in-tree by filtergs_b200/build.py.  There is no fallback:
if the shared library is missing or does not load, every entry point raises.
"""
import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libfiltergs_b200.so")

FGS_OK = 0
FGS_ERR_ARG = 1
FGS_ERR_CUDA = 2
FGS_ERR_TIMEOUT = 3
FGS_ERR_PREFILTERED = 4
FGS_ERR_CAPACITY = 5
FGS_ERR_OVERFLOW = 6
FGS_BACKWARD_REF_COMPAT = 0
FGS_BACKWARD_CONSISTENT = 1
FGS_STATS_SLOTS = 64

vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float
i64 = C.c_longlong
sz = C.c_size_t


class RasterArgs(C.Structure):
    """Mirror of struct fgs_raster_args."""
    _fields_ = [
        ("P", i32), ("D", i32), ("M", i32), ("width", i32), ("height", i32),
        ("background", vp), ("means3D", vp), ("shs", vp), ("colors_precomp", vp), ("opacities", vp),
        ("scales", vp), ("scale_modifier", f32), ("rotations", vp), ("cov3D_precomp", vp),
        ("viewmatrix", vp), ("projmatrix", vp), ("campos", vp), ("tan_fovx", f32), ("tan_fovy", f32),
        ("prefiltered", i32), ("use_filter", i32),
        ("ogfs_epsilon_scale", f32), ("ogfs_epsilon_max", f32), ("ogfs_energy_floor", f32),
        ("ogfs_radius_ratio_min", f32), ("ogfs_enable_stats", i32), ("filter3d_scale", f32),
    ]


class AdamArgs(C.Structure):
    """Mirror of struct fgs_adam_args."""
    _fields_ = [("P", i32), ("M", i32), ("lr", f32 * 5), ("beta1", C.c_double), ("beta2", C.c_double),
                ("eps", f32)] + [
        (n, vp) for n in ("xyz", "shs", "opac_logit", "log_scale", "rot_raw", "opac", "scale", "rot",
                          "g_xyz", "g_shs", "g_opac", "g_scale", "g_rot",
                          "m_xyz", "m_shs", "m_opac", "m_scale", "m_rot",
                          "v_xyz", "v_shs", "v_opac", "v_scale", "v_rot")]


# name -> (restype, argtypes)
SIGNATURES = {
    "fgs_status_string": (C.c_char_p, [i32]),
    "fgs_version": (C.c_char_p, []),
    "fgs_geom_bytes": (sz, [i32]),
    "fgs_image_bytes": (sz, [i32, i32]),
    "fgs_binning_bytes": (sz, [i64, i32]),
    "fgs_forward_preprocess": (i32, [C.POINTER(RasterArgs), vp, vp, vp, C.POINTER(i64), vp]),
    "fgs_forward_render": (i32, [C.POINTER(RasterArgs), vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, i32, vp]),
    "fgs_backward": (i32, [C.POINTER(RasterArgs), vp, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                           i32, vp]),
    "fgs_check": (i32, [vp, vp]),
    "fgs_mark_visible": (i32, [i32, vp, vp, vp, vp, vp]),
    "fgs_compute_radius": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, f32, f32, vp, vp]),
    "fgs_compute_radius_v2": (i32, [i32, vp, vp, vp, vp, vp, f32, f32, f32, f32, vp, vp]),
    "fgs_visibility_radius": (i32, [i32, vp, vp, vp, vp, vp, vp, vp, i32, f32, f32, f32, f32, f32, f32, f32,
                                    vp, vp, vp, vp]),
    "fgs_sorted_pairs": (i32, [vp, vp, i32, i64, vp, vp, vp]),
    "fgs_preprocess_outputs": (i32, [vp, i32, vp, vp, vp, vp, vp, vp]),
    "fgs_image_outputs": (i32, [vp, i32, i32, vp, vp, vp, vp]),
    "fgs_profile_enable": (i32, [i32]),
    "fgs_profile_read": (i32, [vp, vp, i32]),
    "fgs_launch_count": (i64, []),
    "fgs_noalloc_capacity_bytes": (sz, []),
    "fgs_debug_lookback_fault": (i32, [C.c_uint, C.c_ulonglong]),
    "fgs_set_render_config": (i32, [i32, i32, i32, i32]),
    "fgs_gather_attributes": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "fgs_compact_scratch_bytes": (sz, [i32]),
    "fgs_compact_mask": (i32, [i32, vp, vp, vp, vp, vp]),
    "fgs_gather_activate": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "fgs_rows_valid": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, vp]),
    "fgs_radius_raw": (i32, [i32, vp, vp, vp, vp, vp, f32, f32, f32, f32, vp, vp]),
    "fgs_log_cut_scratch_bytes": (sz, [i32, i32, i32, i32]),
    "fgs_log_cut": (i32, [i32, vp, i32, vp, vp, i32, vp, f32, i32, vp, vp, vp, vp]),
    "fgs_cull": (i32, [vp, vp, i32, vp, vp, f32, vp, vp, vp, vp]),
    "fgs_ancestor_path": (i32, [i32, vp, vp, i32, vp, vp, vp]),
    "fgs_batch_workspace_bytes": (sz, [i32, i32, vp]),
    "fgs_batch_create": (vp, [C.POINTER(RasterArgs), i32, vp, vp, sz, i32, vp, vp, vp, vp, vp, C.POINTER(i32), vp]),
    "fgs_batch_forward": (i32, [vp, vp]),
    "fgs_batch_backward": (i32, [vp, vp]),
    "fgs_batch_set_view_io": (i32, [vp, i32, vp, vp, vp, vp]),
    "fgs_batch_set_view_outputs": (i32, [vp, i32, vp, vp, vp, vp, vp]),
    "fgs_batch_pair_counts": (i32, [vp, vp, vp]),
    "fgs_batch_check": (i32, [vp, vp]),
    "fgs_batch_destroy": (None, [vp]),
    "fgs_batch_set_densify": (i32, [vp, vp, vp, vp]),
    "fgs_loss_scratch_bytes": (sz, [i32, i32]),
    "fgs_loss_l1_ssim": (i32, [i32, i32, vp, vp, vp, f32, f32, vp, vp, vp]),
    "fgs_train_activate": (i32, [i32, vp, vp, vp, vp, vp, vp, vp]),
    "fgs_densify_dense": (i32, [i32, vp, vp, vp, vp, vp, vp]),
    "fgs_adam_step": (i32, [C.POINTER(AdamArgs), vp, vp, vp]),
    "fgs_get_render_config": (i32, [vp]),
    "fgs_set_render_split": (i32, [i32, i32]),
    "fgs_get_render_split": (i32, [vp]),
    "fgs_forward_noalloc": (i32, [C.POINTER(RasterArgs), vp, vp, vp, vp, vp, C.POINTER(i64), vp]),
}

STAGES = ["preprocess", "depth_sort", "duplicate", "tile_sort", "ranges", "render_fwd", "stats", "render_bwd",
          "preprocess_bwd"]

_lib = None


class FgsError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        text = status_string(status) if _lib is not None else str(status)
        super().__init__(f"{where}: {text} (status {status})")


def lib():
    """Load the shared library once; raise loudly when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"filtergs_b200 CUDA library not built: {LIB_PATH} is missing "
                               "(run `python -m filtergs_b200.build`)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(status):
    return lib().fgs_status_string(int(status)).decode()


def check(status, where):
    if status != FGS_OK:
        raise FgsError(status, where)


def profile_enable(on=True):
    lib().fgs_profile_enable(int(bool(on)))


def profile_read(reset=True):
    """Per-stage (milliseconds summed, calls) recorded since the last reset."""
    import numpy as np
    ms = np.zeros(len(STAGES), np.float64)
    calls = np.zeros(len(STAGES), np.int64)
    check(lib().fgs_profile_read(ms.ctypes.data_as(vp), calls.ctypes.data_as(vp), int(bool(reset))),
          "fgs_profile_read")
    return {n: (float(ms[i]), int(calls[i])) for i, n in enumerate(STAGES)}


def set_render_config(fwd_ppt=2, fwd_batch=256, bwd_ppt=2, bwd_batch=256):
    check(lib().fgs_set_render_config(int(fwd_ppt), int(fwd_batch), int(bwd_ppt), int(bwd_batch)),
          "fgs_set_render_config")


BAND_SHAPES = {0: (16, 2), 1: (8, 4), 2: (4, 4), 3: (4, 2)}


def set_render_split(min_records=0, band_shape=0):
    """Forward tiles with at least min_records pairs are rendered in bands (0: never) of
    BAND_SHAPES[band_shape] pixels, one warp each."""
    check(lib().fgs_set_render_split(int(min_records), int(band_shape)), "fgs_set_render_split")


def get_render_split():
    """(min_records, band_shape) of the forward's long-tile bands."""
    cfg = (C.c_int * 2)()
    check(lib().fgs_get_render_split(C.cast(cfg, vp)), "fgs_get_render_split")
    return int(cfg[0]), int(cfg[1])


def get_render_config():
    cfg = (C.c_int * 4)()
    check(lib().fgs_get_render_config(C.cast(cfg, vp)), "fgs_get_render_config")
    return tuple(cfg)


def launch_count():
    return int(lib().fgs_launch_count())


def call(name, *args):
    """Call an int-returning entry point and raise FgsError on failure."""
    st = getattr(lib(), name)(*args)
    check(st, name)
    return st
