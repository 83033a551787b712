"""The binning-tile study: why the autotuner keeps the reference's 16x16 tile.

The C oracle is built with 8x8 and 16x8 binning tiles (oracle.build_tile_variant;
lambda_G's exponent kept at the reference's 256, forward.cu:348) and its images and
pair counts are compared with the 16x16 build on the same views.  A Gaussian reaches
every pixel of every tile its rectangle covers (getRect rounds the OGFS radius out to
tile boundaries, auxiliary.h), so a smaller tile drops the contributions of pixels
between the radius and the 16-pixel tile edge: the image changes, and the pairs to
sort and composite grow.  Asserted here on a small aerial view; the headline-size
figures (2M Gaussians, two 1920x1080 cameras of the benchmark's sequence) are printed
with FGS_TILE_SHAPE_FULL=1:

    FGS_TILE_SHAPE_FULL=1 python -m pytest tests/test_tile_shape_cpu.py -s -q
"""
import os

import numpy as np
import pytest

from filtergs_b200 import synthetic as S
from oracle import oracle as O


def _view(sc, cam):
    return O.Scene(sc["means3D"], sc["opacities"], cam.W, cam.H, cam.tanfovx, cam.tanfovy,
                   cam.viewmatrix.reshape(-1), cam.projmatrix.reshape(-1), cam.campos, shs=sc["shs"], sh_degree=3,
                   scales=sc["scales"], rotations=sc["rotations"])


def _render(lib, tile, s):
    pre = O.preprocess(s, lib=lib)
    _, vals, ranges = O.bin_pairs(pre, s.W, s.H, lib=lib, tile=tile)
    return O.render(s, pre, vals, ranges, lib=lib)["color"], len(vals)


def _study(sc, cams, tmp):
    libs = {t: O.build_tile_variant(*t, tmp) for t in ((16, 16), (8, 8), (16, 8))}
    rows = []
    for cam in cams:
        s = _view(sc, cam)
        base, k0 = _render(libs[(16, 16)], (16, 16), s)
        ref_img = O.forward(s)["color"]  # the default build: the 16x16 variant must equal it
        assert np.array_equal(base, ref_img)
        for t in ((8, 8), (16, 8)):
            img, k = _render(libs[t], t, s)
            d = np.abs(img - base)
            mse = float(np.mean((img - base) ** 2))
            rows.append(dict(tile=t, pairs=k, pairs_16x16=k0, changed=float((d > 1e-5).mean()),
                             max_abs=float(d.max()), psnr=10 * np.log10(1.0 / mse) if mse > 0 else float("inf")))
    return rows


def test_smaller_binning_tiles_change_the_image_and_add_pairs(tmp_path):
    sc = S.urban_scene(P=200_000, seed=1001, half_extent=150.0, buildings=40)
    rng = np.random.default_rng(2001)
    cams = [S.aerial_camera(rng, W=640, H=360, fx=1600.0 * 640 / 1920, xy_range=100.0)]
    rows = _study(sc, cams, str(tmp_path))
    by = {r["tile"]: r for r in rows}
    small, mid = by[(8, 8)], by[(16, 8)]
    assert small["pairs"] > 1.5 * small["pairs_16x16"]
    assert small["pairs_16x16"] < mid["pairs"] < small["pairs"]
    assert small["changed"] > 0.05 and mid["changed"] > 0.02
    assert small["changed"] > mid["changed"]


@pytest.mark.skipif(not os.environ.get("FGS_TILE_SHAPE_FULL"), reason="headline-size study: FGS_TILE_SHAPE_FULL=1")
def test_tile_study_at_headline_size(tmp_path):
    sc = S.urban_scene(P=2_000_000, seed=1001)
    rng = np.random.default_rng(2001)  # the benchmark's first two 1080p cameras
    cams = [S.aerial_camera(rng, W=1920, H=1080) for _ in range(2)]
    O.set_threads(os.cpu_count())
    for r in _study(sc, cams, str(tmp_path)):
        print(f"{r['tile'][0]}x{r['tile'][1]}: pairs {r['pairs']} vs {r['pairs_16x16']} "
              f"({r['pairs'] / r['pairs_16x16']:.2f}x), values changed > 1e-5 {100 * r['changed']:.1f}%, "
              f"max {r['max_abs']:.3f}, PSNR {r['psnr']:.1f} dB")
