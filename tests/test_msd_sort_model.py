"""The MSD radix sort of the sorted-entry stage, replayed on the CPU (no GPU).

k_msd_count / k_msd_prefix / k_msd_tiles / k_msd_scatter (msm_kernels.cuh)
are restated here index for index: group geometry (pass 1: the tiles of
[0, E) split evenly over the plan's groups, each counted in MSD_COUNT_PARTS
parts; pass 2: chunks of at most MSD_CHUNK_TILES tiles of each pass-1
segment through the tile and chunk tables), the count rows, the group
totals written straight into the [segment][digit][group] scan layout and
its exclusive scan, the slot rows of k_msd_prefix, and each tile's
placement (local digit offsets from its count row plus the slot of its
run).  On random key sets -- uniform, skewed (one bucket holding a fifth of
the entries, like witness scalars equal to 1), with fewer entries than the
plan's bound, and empty -- every index stays inside its buffer, no output
slot is written twice and the result is ordered by bucket id.  Plans (digit
widths, tile and group bounds) come from the real C++ planner through
zkmsm_plan_describe.
"""
import ctypes
import json
import os
import re
import zlib

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
PARTS = _const("MSD_COUNT_PARTS")
CHUNK = _const("MSD_CHUNK_TILES")


def plan(counts, curve=0):
    buf = ctypes.create_string_buffer(1 << 24)
    c = (ctypes.c_uint32 * len(counts))(*counts)
    assert zl.lib().zkmsm_plan_describe(curve, c, len(counts), 1, 0, 0, -1, 0, buf, len(buf)) == 0
    return json.loads(buf.value.decode())


def excl_scan(h):
    out = np.zeros_like(h)
    np.cumsum(h[:-1], out=out[1:])
    return out


def group(u, E, ng, sub, whole, seg_start, seg_tile, seg_chunk, nb):
    """msd_group: (lo, hi, row0, sidx, sstride) of unit u, or None."""
    if seg_chunk is None:
        grp, part = (u, 0) if whole else (u // sub, u % sub)
        if grp >= ng:
            return None
        nt = (E + TILE - 1) // TILE
        K = (nt + ng - 1) // ng
        Ks = (K + sub - 1) // sub
        gend = (grp + 1) * K
        t0, t1 = grp * K, gend
        if not whole:
            t0 += part * Ks
            t1 = min(t0 + Ks, gend)
        t1 = min(t1, nt)
        t0 = min(t0, t1)
        return min(t0 * TILE, E), min(t1 * TILE, E), t0, grp * sub + part, ng * sub
    nseg = len(seg_chunk) - 1
    if u >= seg_chunk[nseg]:
        return None
    a, b = 0, nseg - 1
    while a < b:
        mid = (a + b + 1) >> 1
        if seg_chunk[mid] <= u:
            a = mid
        else:
            b = mid - 1
    k = u - seg_chunk[a]
    lo = seg_start[a] + k * CHUNK * TILE
    end = seg_start[a + 1]
    assert lo < end, "chunk starts past its segment"
    hi = min(end, lo + CHUNK * TILE)
    row0 = seg_tile[a] + k * CHUNK
    assert row0 + (hi - lo + TILE - 1) // TILE <= seg_tile[a + 1], "chunk rows spill into the next segment"
    return lo, hi, row0, seg_chunk[a] * nb + k, seg_chunk[a + 1] - seg_chunk[a]


def tiles_of(g):
    lo, hi, row0 = g[0], g[1], g[2]
    return [(t0, min(t0 + TILE, hi), row0 + j) for j, t0 in enumerate(range(lo, hi, TILE))]


def tile_range(t, E, seg):
    """msd_tile: (lo, hi) of tile t, or None past the pass-2 tiles."""
    if seg is None:
        return min(t * TILE, E), min(t * TILE + TILE, E)
    seg_start, seg_tile, _ = seg
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
    lo = seg_start[a] + (t - seg_tile[a]) * TILE
    assert lo < seg_start[a + 1], "tile starts past its segment"
    return lo, min(seg_start[a + 1], lo + TILE)


def msd_pass(keys, vals, E, shift, bits, ng, sub, ntiles, seg, rows_size, scan_size):
    """One pass as the device runs it: k_msd_count over ng*sub units (count
    rows C[tile][digit], unit totals into the scan layout S), the exclusive
    scan of S over its bound, k_msd_prefix over ng groups (slot rows
    P[tile][digit]), k_msd_scatter over the `ntiles` tile bound (local
    offsets from the tile's C row, run slots from its P row)."""
    nb = 1 << bits
    seg_start, seg_tile, seg_chunk = seg if seg else (None, None, None)
    C = np.full(rows_size, 5, dtype=np.int64)  # stale contents everywhere
    P = np.full(rows_size, 9, dtype=np.int64)
    S = np.full(scan_size, 7, dtype=np.int64)
    used = np.zeros(scan_size, dtype=bool)
    rows_seen = {}
    for u in range(ng * sub):  # k_msd_count
        g = group(u, E, ng, sub, False, seg_start, seg_tile, seg_chunk, nb)
        if g is None:
            continue
        tot = np.zeros(nb, dtype=np.int64)
        for lo, hi, row in tiles_of(g):
            assert (row + 1) * nb <= rows_size and row not in rows_seen
            rows_seen[row] = (lo, hi)
            C[row * nb:(row + 1) * nb] = np.bincount((keys[lo:hi] >> shift) & (nb - 1), minlength=nb)
            tot += C[row * nb:(row + 1) * nb]
        idx = g[3] + np.arange(nb) * g[4]
        assert idx.max() < scan_size and not used[idx].any()
        used[idx] = True
        S[idx] = tot
    n_used = int(used.sum())
    assert used[:n_used].all(), "group totals are not a prefix of the scan layout"
    S[:nb * ng * sub] = excl_scan(S[:nb * ng * sub])  # the scan runs over the bound
    for u in range(ng):  # k_msd_prefix
        g = group(u, E, ng, sub, True, seg_start, seg_tile, seg_chunk, nb)
        if g is None:
            continue
        run = S[g[3] + np.arange(nb) * g[4]].copy()
        for lo, hi, row in tiles_of(g):
            P[row * nb:(row + 1) * nb] = run
            run = run + C[row * nb:(row + 1) * nb]
    outk = np.full(E, -1, dtype=np.int64)
    outv = np.full(E, -1, dtype=np.int64)
    for t in range(ntiles):  # k_msd_scatter
        r = tile_range(t, E, seg)
        if r is None or r[0] == r[1]:
            continue
        lo, hi = r
        assert rows_seen.get(t) == (lo, hi), "rows of tile %d were written for another range" % t
        d = (keys[lo:hi] >> shift) & (nb - 1)
        cnt = C[t * nb:(t + 1) * nb]
        off = excl_scan(cnt)
        perm = np.random.default_rng(lo).permutation(hi - lo)  # any order inside a digit
        order = perm[np.argsort(d[perm], kind="stable")]
        dd = d[order]
        dst = P[t * nb + dd] - off[dd] + np.arange(hi - lo)
        assert (dst >= 0).all() and (dst < E).all() and (outk[dst] == -1).all()
        assert len(np.unique(dst)) == len(dst)
        outk[dst] = keys[lo + order]
        outv[dst] = vals[lo + order]
    assert (outk >= 0).all()
    return outk, outv, S


def msd_tiles(S1, stride1, nseg, E):
    seg_start = [int(S1[s * stride1]) for s in range(nseg)] + [E]
    nt = [(seg_start[s + 1] - seg_start[s] + TILE - 1) // TILE for s in range(nseg)]
    nc = [(t + CHUNK - 1) // CHUNK for t in nt]
    seg_tile = [0] + [int(x) for x in np.cumsum(nt)]
    seg_chunk = [0] + [int(x) for x in np.cumsum(nc)]
    return seg_start, seg_tile, seg_chunk


def run_msd(pl, keys):
    passes, b1, b2, t1, t2, g1, ch2 = pl["msd"]
    E = len(keys)
    assert E <= pl["entry_bound"]
    vals = np.arange(E, dtype=np.int64)
    rows = max((1 << b1) * t1, (1 << b2) * t2 if passes == 2 else 0)
    scan = max((1 << b1) * g1 * PARTS, (1 << b2) * ch2 if passes == 2 else 0)
    shift1 = b2 if passes == 2 else 0
    k1, v1, S1 = msd_pass(keys, vals, E, shift1, b1, g1, PARTS, t1, None, rows, scan)
    if passes == 1:
        return k1, v1
    seg = msd_tiles(S1, g1 * PARTS, 1 << b1, E)
    assert seg[1][-1] <= t2, "pass-2 tiles exceed the count rows"
    assert seg[2][-1] <= ch2, "pass-2 chunks exceed the bound the grid is launched for"
    return msd_pass(k1, v1, E, 0, b2, ch2, 1, t2, seg, rows, scan)[:2]


@pytest.mark.parametrize("counts", [[1 << 20], [1 << 24], [(1 << 21) + 77], [4096, 1 << 20, 333, 1 << 19]])
def test_plans_choose_msd_within_limits(counts):
    pl = plan(counts)
    passes, b1, b2, t1, t2, g1, ch2 = pl["msd"]
    kb = max(1, (pl["nbuckets"] - 1).bit_length())
    assert passes in (1, 2) and b1 + b2 == kb and max(b1, b2) <= MAX_BITS
    assert t1 * TILE >= pl["entry_bound"]
    assert 1 <= g1 <= min(t1, 148)
    if passes == 2:
        assert t2 == t1 + (1 << b1)
        assert ch2 == (t2 + CHUNK - 1) // CHUNK + (1 << b1)


@pytest.mark.parametrize("case", ["uniform", "hot", "sparse", "empty"])
def test_msd_sort_replay(case):
    pl = plan([1 << 19])  # a real two-pass plan (18-bit bucket ids)
    assert pl["msd"][0] == 2
    G = pl["nbuckets"]
    rng = np.random.default_rng(zlib.crc32(case.encode()))
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
