"""bench.py's roofline bookkeeping on the CPU: which launch is the dominant kernel,
its algorithmic bytes, and the issue-roof figure built from the committed ncu
summary.  Stage times are given as (summed event ms, launches), as the bench's
per-stage profile reports them."""
from types import SimpleNamespace

import pytest

import bench

# one batched step of 16 views: the per-view front-end stages overlap on the
# front-end streams, so their summed event times can exceed a compositing launch's
PROF = {"preprocess": (149.4, 340), "tile_sort": (196.3, 320), "render_fwd": (117.5, 20),
        "render_bwd": (189.9, 20), "preprocess_bwd": (27.8, 20)}
VIEWS = [{"cam": SimpleNamespace(W=1920, H=1080)}] * 16
K, V = [2_360_215] * 16, [118_117] * 16


def test_batched_dominant_kernel_is_a_launch_that_runs_alone():
    r = bench.roofline(PROF, 2_000_000, VIEWS, K, V, batched=True)
    assert r["kernel"] == "render_bwd"
    # 40 K + 20 N + 44 V per view, summed over the views one launch covers
    assert r["algorithmic_bytes_per_launch"] == 16 * (40 * K[0] + 20 * 1920 * 1080 + 44 * V[0])
    assert r["launch_ms"] == pytest.approx(189.9 / 20)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])


def test_plain_dominant_kernel_is_the_largest_stage():
    r = bench.roofline(PROF, 2_000_000, VIEWS[:1], K[:1], V[:1], batched=False)
    assert r["kernel"] == "tile_sort"
    assert r["issue"]["frac"] is None and "tile_sort" in r["issue"]["source"]


def test_issue_roof_is_instructions_over_time_against_four_per_sm_cycle():
    iss = bench.issue_roof("batched.render_bwd", 1e6, 1.0)
    if iss["frac"] is None:  # the summary was captured from other kernel sources
        assert "other kernel sources" in iss["source"]
        return
    assert iss["peak"] == pytest.approx(148 * 4 * 1.965)
    assert iss["achieved"] == pytest.approx(iss["warp_inst_per_launch"] / 1e-3 / 1e9)
    assert 100 < iss["warp_inst_per_launch"] / 1e6 < 400  # warp instructions per pair
