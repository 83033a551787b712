"""CPU: the C-ABI library loads, exports every entry point include/*.h
declares, and validates arguments before touching the GPU."""
import ctypes as C
import glob
import os
import re

import pytest

from filtergs_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(fgs_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _declared()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    # and the ctypes signatures cover them all
    assert set(declared) <= set(_lib.SIGNATURES), sorted(set(declared) - set(_lib.SIGNATURES))


def test_status_strings_and_version():
    assert _lib.status_string(_lib.FGS_OK) == "ok"
    for code in range(1, 7):
        assert _lib.status_string(code) not in ("", "unknown status")
    assert b"sm_100a" in _lib.lib().fgs_version()


def test_workspace_sizes():
    L = _lib.lib()
    g1, g2 = L.fgs_geom_bytes(1000), L.fgs_geom_bytes(2000)
    assert 0 < g1 < g2 and g1 % 256 == 0
    # per Gaussian: 48 B record + radii, tiles, clamp, keys, sort scratch
    assert L.fgs_geom_bytes(1 << 20) >= 73 * (1 << 20)
    assert L.fgs_image_bytes(1920, 1080) >= 8 * 1920 * 1080 + 8 * 120 * 68
    assert L.fgs_binning_bytes(10**6, 1000) >= 64 * 10**6
    assert L.fgs_image_bytes(0, 10) == 0 and L.fgs_geom_bytes(-1) == 0


def test_argument_validation_without_gpu():
    L = _lib.lib()
    K = C.c_longlong(0)
    # null argument block
    assert L.fgs_forward_preprocess(None, None, None, None, C.byref(K), None) == _lib.FGS_ERR_ARG
    a = _lib.RasterArgs()
    a.P, a.width, a.height = 10, 0, 16
    assert L.fgs_forward_preprocess(C.byref(a), None, None, None, C.byref(K), None) == _lib.FGS_ERR_ARG
    a.width = 16                               # no means / opacities / matrices
    assert L.fgs_forward_preprocess(C.byref(a), None, None, None, C.byref(K), None) == _lib.FGS_ERR_ARG
    assert L.fgs_backward(C.byref(a), None, None, None, 0, None, None, None, None, None, None, None, None, None,
                          None, None, 7, None) == _lib.FGS_ERR_ARG
    assert L.fgs_set_render_config(3, 64, 2, 64) == _lib.FGS_ERR_ARG
    assert L.fgs_set_render_config(2, 96, 2, 64) == _lib.FGS_ERR_ARG
    assert L.fgs_mark_visible(-1, None, None, None, None, None) == _lib.FGS_ERR_ARG
    assert L.fgs_visibility_radius(5, None, None, None, None, None, None, None, 4, 1, 1, 1, 1, 0.1, 1.5, 700,
                                   None, None, None, None) == _lib.FGS_ERR_ARG


def test_render_config_roundtrip():
    old = _lib.get_render_config()
    try:
        _lib.set_render_config(4, 128, 1, 64)
        assert _lib.get_render_config() == (4, 128, 1, 64)
    finally:
        _lib.set_render_config(*old)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError, match="not built"):
        _lib.lib()


def test_batch_workspace_planning():
    """fgs_batch_workspace_bytes (host only): per view one geom + image + binning at its pair
    capacity and 11 floats of screen-space scratch per Gaussian; per batch one bit per view per
    Gaussian in 32-view words and the list of Gaussians some view saw."""
    from filtergs_b200.batched import _ViewArgs
    L = _lib.lib()
    P = 100_000

    def size(n, W=64, H=48, cap=5000):
        va = (_ViewArgs * n)()
        for v in va:
            v.width, v.height, v.pair_capacity = W, H, cap
        return int(L.fgs_batch_workspace_bytes(P, n, C.cast(va, C.c_void_p)))

    per_view = L.fgs_geom_bytes(P) + L.fgs_image_bytes(64, 48) + L.fgs_binning_bytes(5000, P) + 44 * P
    s1, s32, s33 = size(1), size(32), size(33)
    assert s1 >= per_view + 4 * P + 4 * P            # one view-bit word and the seen list
    assert s32 - s1 >= 31 * per_view
    # the 33rd view adds its own state and a second word of view bits
    assert s33 - s32 >= per_view + 4 * P
    assert size(2, cap=10_000) > size(2, cap=5000)
    assert size(0) == 0
    va = (_ViewArgs * 1)()
    va[0].width, va[0].height, va[0].pair_capacity = 0, 48, 10
    assert L.fgs_batch_workspace_bytes(P, 1, C.cast(va, C.c_void_p)) == 0
