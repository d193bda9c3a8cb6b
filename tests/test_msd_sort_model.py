"""The MSD radix sort of the sorted-entry stage, replayed on the CPU (no GPU).

k_msd_count / k_msd_transpose / k_msd_tiles / k_msd_scatter (msm_kernels.cuh)
are restated here index for index: tile geometry (pass 1 over [0, E); pass 2
over the pass-1 segments through the tile table), the count rows, the
[segment][digit][tile] scan layout and its exclusive scan, the slot rows, and
each tile's placement (local digit offsets from its count row plus the slot
of its run).  On random key sets -- uniform,
skewed (one bucket holding a fifth of the entries, like witness scalars
equal to 1), with fewer entries than the plan's bound, and empty -- every
index stays inside its buffer, no output slot is written twice and the
result is ordered by bucket id.  Plans (digit widths, tile bounds) come from
the real C++ planner through zkmsm_plan_describe.
"""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from zkmetal_b200 import lib as zl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _const(name):
    text = open(os.path.join(ROOT, "zkmetal_b200", "csrc", "types.cuh")).read()
    m = re.search(r"constexpr\s+\w+\s+%s\s*=\s*([^;]+);" % name, text)
    return int(eval(m.group(1).replace("ull", "")))


TILE = _const("MSD_TILE")
MAX_BITS = _const("MSD_MAX_BITS")


def plan(counts, curve=0):
    buf = ctypes.create_string_buffer(1 << 24)
    c = (ctypes.c_uint32 * len(counts))(*counts)
    assert zl.lib().zkmsm_plan_describe(curve, c, len(counts), 1, 0, 0, -1, 0, buf, len(buf)) == 0
    return json.loads(buf.value.decode())


def excl_scan(h):
    out = np.zeros_like(h)
    np.cumsum(h[:-1], out=out[1:])
    return out


def geom(t, E, ntiles, seg_start, seg_tile, nb):
    if seg_tile is None:
        if t >= ntiles:
            return None
        lo = min(t * TILE, E)
        return lo, min(lo + TILE, E), t, ntiles, 0
    nseg = len(seg_tile) - 1
    if t >= seg_tile[nseg]:
        return None
    a, b = 0, nseg - 1
    while a < b:
        mid = (a + b + 1) >> 1
        if seg_tile[mid] <= t:
            a = mid
        else:
            b = mid - 1
    k = t - seg_tile[a]
    nt = seg_tile[a + 1] - seg_tile[a]
    lo = seg_start[a] + k * TILE
    assert lo < seg_start[a + 1], "tile starts past its segment"
    return lo, min(seg_start[a + 1], lo + TILE), k, nt, seg_tile[a] * nb


def msd_pass(keys, vals, E, shift, bits, ntiles, seg_start, seg_tile, hsize, grid):
    """One pass as the device runs it: k_msd_count (rows C[tile][digit]),
    k_msd_transpose to the scan layout S, the exclusive scan, the transpose
    back to slot rows P, k_msd_scatter (local offsets from the tile's C row,
    run slots from its P row)."""
    nb = 1 << bits
    C = np.full(hsize, 5, dtype=np.int64)  # stale contents everywhere
    S = np.full(hsize, 7, dtype=np.int64)
    P = np.full(hsize, 9, dtype=np.int64)
    geoms = [geom(t, E, ntiles, seg_start, seg_tile, nb) for t in range(grid)]
    for t, g in enumerate(geoms):  # k_msd_count
        if g is None:
            continue
        lo, hi, k, nt, hb = g
        assert (t + 1) * nb <= hsize
        C[t * nb:(t + 1) * nb] = np.bincount((keys[lo:hi] >> shift) & (nb - 1), minlength=nb)
    used = np.zeros(hsize, dtype=bool)
    for t, g in enumerate(geoms):  # k_msd_transpose, rows -> scan layout
        if g is None:
            continue
        lo, hi, k, nt, hb = g
        idx = hb + np.arange(nb) * nt + k
        assert idx.max() < hsize and not used[idx].any()
        used[idx] = True
        S[idx] = C[t * nb:(t + 1) * nb]
    n_used = int(used.sum())
    assert used[:n_used].all(), "pass counts are not a prefix of the scan layout"
    S[:grid * nb] = excl_scan(S[:grid * nb])  # the scan runs over the bound
    for t, g in enumerate(geoms):  # k_msd_transpose back, scan layout -> slot rows
        if g is None:
            continue
        lo, hi, k, nt, hb = g
        P[t * nb:(t + 1) * nb] = S[hb + np.arange(nb) * nt + k]
    outk = np.full(E, -1, dtype=np.int64)
    outv = np.full(E, -1, dtype=np.int64)
    for t, g in enumerate(geoms):  # k_msd_scatter
        if g is None or g[0] == g[1]:
            continue
        lo, hi, k, nt, hb = g
        d = (keys[lo:hi] >> shift) & (nb - 1)
        off = excl_scan(C[t * nb:(t + 1) * nb])
        perm = np.random.default_rng(t).permutation(hi - lo)  # any order inside a digit
        order = perm[np.argsort(d[perm], kind="stable")]
        dd = d[order]
        dst = P[t * nb + dd] - off[dd] + np.arange(hi - lo)
        assert (dst >= 0).all() and (dst < E).all() and (outk[dst] == -1).all()
        assert len(np.unique(dst)) == len(dst)
        outk[dst] = keys[lo + order]
        outv[dst] = vals[lo + order]
    assert (outk >= 0).all()
    return outk, outv, S


def msd_tiles(Hs, ntiles1, nseg, E):
    seg_start = [int(Hs[s * ntiles1]) for s in range(nseg)] + [E]
    nt = [(seg_start[s + 1] - seg_start[s] + TILE - 1) // TILE for s in range(nseg)]
    seg_tile = [0] + list(np.cumsum(nt))
    return seg_start, [int(x) for x in seg_tile]


def run_msd(pl, keys):
    passes, b1, b2, t1, t2 = pl["msd"]
    E = len(keys)
    assert E <= pl["entry_bound"]
    vals = np.arange(E, dtype=np.int64)
    hsize = max((1 << b1) * t1, (1 << b2) * t2 if passes == 2 else 0)
    shift1 = b2 if passes == 2 else 0
    k1, v1, Hs = msd_pass(keys, vals, E, shift1, b1, t1, None, None, hsize, t1)
    if passes == 1:
        return k1, v1
    seg_start, seg_tile = msd_tiles(Hs, t1, 1 << b1, E)
    assert seg_tile[-1] <= t2, "pass-2 tiles exceed the bound the grid is launched for"
    return msd_pass(k1, v1, E, 0, b2, 0, seg_start, seg_tile, hsize, t2)[:2]


@pytest.mark.parametrize("counts", [[1 << 20], [1 << 24], [(1 << 21) + 77], [4096, 1 << 20, 333, 1 << 19]])
def test_plans_choose_msd_within_limits(counts):
    pl = plan(counts)
    passes, b1, b2, t1, t2 = pl["msd"]
    kb = max(1, (pl["nbuckets"] - 1).bit_length())
    assert passes in (1, 2) and b1 + b2 == kb and max(b1, b2) <= MAX_BITS
    assert t1 * TILE >= pl["entry_bound"]
    if passes == 2:
        assert t2 == t1 + (1 << b1)


@pytest.mark.parametrize("case", ["uniform", "hot", "sparse", "empty"])
def test_msd_sort_replay(case):
    pl = plan([1 << 19])  # a real two-pass plan (18-bit bucket ids)
    assert pl["msd"][0] == 2
    G = pl["nbuckets"]
    rng = np.random.default_rng(hash(case) & 0xFFFF)
    bound = pl["entry_bound"]
    if case == "uniform":
        E = bound - 12345
        keys = rng.integers(0, G, E)
    elif case == "hot":
        E = bound // 3
        keys = rng.integers(0, G, E)
        keys[rng.random(E) < 0.2] = 0  # a fifth of the entries in bucket 0
    elif case == "sparse":
        E = 5000
        keys = rng.integers(0, G, E)
    else:
        E = 0
        keys = np.zeros(0, dtype=np.int64)
    keys = keys.astype(np.int64)
    k, v = run_msd(pl, keys)
    assert (np.diff(k) >= 0).all()
    assert sorted(v.tolist()) == list(range(E)) and (keys[v] == k).all()
