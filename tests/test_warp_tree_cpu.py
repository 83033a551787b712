"""The nine-value warp reduction of the backward (warp_transpose_sum9 in
csrc/fgs_common.cuh), replayed lane by lane on the CPU: after its levels
(9 -> 5/4 -> 3/2 -> 2/1 -> 1 values per lane, partners at lane distance 16, 8, 4,
2, then a butterfly step at distance 1) every lane must hold the warp total of
the component that sum9_component's table names for it, and the even lanes must
cover the nine components once each.  The table is read from the header, so a
change to the split without the table (or the reverse) fails here.
"""
import os
import re

import numpy as np

HDR = os.path.join(os.path.dirname(__file__), "..", "filtergs_b200", "csrc", "fgs_common.cuh")
LANES = np.arange(32)


def _level(vals, keep, dist):
    """sum9_level<keep, len(vals)>: lanes with bit `dist` clear keep values [0, keep)."""
    hi = (LANES & dist) != 0
    out = []
    for i in range(keep):
        lo_v = vals[i]
        hi_v = vals[i + keep] if i + keep < len(vals) else np.zeros(32)
        send = np.where(hi, lo_v, hi_v)
        kept = np.where(hi, hi_v, lo_v)
        out.append(kept + send[LANES ^ dist])
    return out


def _table():
    src = open(HDR).read()
    body = src[src.index("int sum9_component"):]
    m = re.search(r"0x([0-9a-fA-F]+)ull", body)
    assert m, "sum9_component's table constant not found"
    t = int(m.group(1), 16)
    return [(t >> (4 * (lane >> 1))) & 15 for lane in range(32)]


def test_warp_tree_lanes_hold_their_component_totals():
    rng = np.random.default_rng(7)
    g = rng.integers(-1000, 1000, size=(32, 9)).astype(np.float64)  # exact sums
    vals = [g[:, q] for q in range(9)]
    for keep, dist in ((5, 16), (3, 8), (2, 4), (1, 2)):
        vals = _level(vals, keep, dist)
    res = vals[0] + vals[0][LANES ^ 1]
    tot = g.sum(axis=0)
    table = _table()
    for lane in range(32):
        q = table[lane]
        if q < 9:
            assert res[lane] == tot[q], (lane, q)
    assert sorted(table[lane] for lane in range(0, 32, 2) if table[lane] < 9) == list(range(9))
