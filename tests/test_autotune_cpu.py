"""CPU: the launch-shape autotuner's host logic (filtergs_b200/autotune.py) on a synthetic cost
table: it installs the fastest forward and the fastest backward shape independently, then the
fastest long-tile split with that forward shape, restores nothing it should not, and answers a
repeated key from its cache without running the step again.  The library's configuration calls
are host-only; the stage timer and the device synchronisation are replaced by fakes."""
import pytest
import torch

from filtergs_b200 import _lib, autotune

FWD = {(1, 64): 9.0, (1, 128): 8.5, (1, 256): 8.2, (2, 64): 6.1, (2, 128): 5.9, (2, 256): 7.2,
       (4, 64): 5.8, (4, 128): 6.0, (4, 256): 6.4}
BWD = {(1, 64): 17.0, (1, 128): 16.7, (1, 256): 16.4, (2, 64): 11.5, (2, 128): 11.3, (2, 256): 15.0,
       (4, 64): 10.1, (4, 128): 10.5, (4, 256): 12.0}
SPLIT = {(0, 0): 0.0, (512, 0): 0.4, (4096, 2): -0.05}


@pytest.fixture
def fake_timer(monkeypatch):
    try:
        saved = _lib.get_render_config(), _lib.get_render_split()
    except Exception as e:  # the library is not built: nothing to test on this machine
        pytest.skip(f"library unavailable: {e}")
    state = {"steps": 0, "pending": [0.0, 0.0]}
    stages = list(_lib.STAGES)

    def run_step():
        fp, fb, bp, bb = _lib.get_render_config()
        state["steps"] += 1
        state["pending"][0] += FWD[(fp, fb)] + SPLIT[tuple(_lib.get_render_split())]
        state["pending"][1] += BWD[(bp, bb)]

    def profile_read(reset=True):
        out = {k: (0.0, 0) for k in stages}
        out["render_fwd"] = (state["pending"][0], 1)
        out["render_bwd"] = (state["pending"][1], 1)
        if reset:
            state["pending"] = [0.0, 0.0]
        return out

    monkeypatch.setattr(_lib, "profile_read", profile_read)
    monkeypatch.setattr(_lib, "profile_enable", lambda on=True: None)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(autotune, "_cache", {})
    yield run_step, state
    _lib.set_render_config(*saved[0])
    _lib.set_render_split(*saved[1])


def test_picks_forward_and_backward_independently(fake_timer):
    run_step, state = fake_timer
    best, table = autotune.tune_render(run_step, key=("w", 1), steps=2, warmup=1,
                                       splits=((0, 0), (512, 0), (4096, 2)))
    assert best == (4, 64, 4, 64)
    assert _lib.get_render_config() == (4, 64, 4, 64)
    assert _lib.get_render_split() == (4096, 2)          # the cheapest split with that forward
    for (p, b), (f, bw) in ((k, v) for k, v in table.items() if k[0] != "split"):
        assert f == pytest.approx(FWD[(p, b)]) and bw == pytest.approx(BWD[(p, b)])
    assert table[("split", 512, 0)][0] == pytest.approx(FWD[(4, 64)] + 0.4)
    # cached: no step runs, the same configuration is installed again
    _lib.set_render_config(1, 64, 1, 64)
    _lib.set_render_split(0, 0)
    n = state["steps"]
    best2, _ = autotune.tune_render(run_step, key=("w", 1))
    assert best2 == best and state["steps"] == n
    assert _lib.get_render_config() == (4, 64, 4, 64) and _lib.get_render_split() == (4096, 2)


def test_mixed_best_shapes(fake_timer, monkeypatch):
    run_step, _ = fake_timer
    monkeypatch.setitem(FWD, (2, 128), 5.0)              # forward now fastest at (2, 128)
    best, _ = autotune.tune_render(run_step, key=("w", 2), steps=1, warmup=0)
    assert best == (2, 128, 4, 64)
    assert _lib.get_render_split() == (0, 0)


def test_invalid_configuration_is_rejected(fake_timer):
    with pytest.raises(_lib.FgsError):
        _lib.set_render_config(3, 64, 4, 64)
    with pytest.raises(_lib.FgsError):
        _lib.set_render_config(4, 96, 4, 64)
    with pytest.raises(_lib.FgsError):
        _lib.set_render_split(-1, 0)
