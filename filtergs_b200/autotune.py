"""Autotuner for the compositing kernels' launch shape.

Sweeps pixels per thread {1, 2, 4} x records per shared-memory batch
{64, 128, 256} for the forward and the backward render kernels on a caller's
own step (one forward + backward on representative views), timing each with
the library's per-stage CUDA events, and installs the fastest pair for the
process (fgs_set_render_config); then, with that shape, the forward's
long-tile threshold among the caller's candidates (fgs_set_render_split).
Results are cached per workload key.
"""
import torch

from . import _lib

PPT = (1, 2, 4)
BATCH = (64, 128, 256)
_cache = {}


def tune_render(run_step, key=None, steps=3, warmup=1, splits=((0, 0),)):
    """run_step() performs one forward + backward through this library.

    splits: candidate (min_records, band_shape) long-tile settings of the forward
    (fgs_set_render_split), tried with the best forward shape; the fastest is installed
    (table keys ("split", min_records, band_shape)).
    Returns ((fwd_ppt, fwd_batch, bwd_ppt, bwd_batch), {(ppt, batch): (fwd_ms, bwd_ms)})."""
    if key is not None and key in _cache:
        best, table, split = _cache[key]
        _lib.set_render_config(*best)
        _lib.set_render_split(*split)
        return best, table
    table = {}
    was = _lib.get_render_config()
    _lib.set_render_split(*splits[0])
    for p in PPT:
        for b in BATCH:
            _lib.set_render_config(p, b, p, b)
            for _ in range(warmup):
                run_step()
            torch.cuda.synchronize()
            _lib.profile_read(reset=True)
            _lib.profile_enable(True)
            for _ in range(steps):
                run_step()
            torch.cuda.synchronize()
            _lib.profile_enable(False)
            prof = _lib.profile_read(reset=True)
            table[(p, b)] = (prof["render_fwd"][0] / steps, prof["render_bwd"][0] / steps)
    if not table:
        _lib.set_render_config(*was)
        return was, table
    bf = min(table, key=lambda c: table[c][0])
    bb = min(table, key=lambda c: table[c][1])
    best = (bf[0], bf[1], bb[0], bb[1])
    _lib.set_render_config(*best)
    split_was = _lib.get_render_split()
    best_split, best_ms = split_was, None
    for sp in splits:
        _lib.set_render_split(*sp)
        ms = _time_fwd(run_step, steps, warmup)
        table[("split",) + tuple(sp)] = (ms, 0.0)
        if best_ms is None or ms < best_ms:
            best_split, best_ms = sp, ms
    _lib.set_render_split(*best_split)
    if key is not None:
        _cache[key] = (best, table, best_split)
    return best, table


def _time_fwd(run_step, steps, warmup):
    for _ in range(warmup):
        run_step()
    torch.cuda.synchronize()
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    for _ in range(steps):
        run_step()
    torch.cuda.synchronize()
    _lib.profile_enable(False)
    return _lib.profile_read(reset=True)["render_fwd"][0] / steps
