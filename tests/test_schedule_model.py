"""CPU model of the device schedule, driven by the library's real host plan.

The plan (window widths, bucket layout, segmented-sum chunking, reduction
tree) comes from the C++ planner through zkmsm_plan_describe.  The kernels'
index logic -- histogram, exclusive scan, counting-sort scatter (in a
shuffled order, as atomics allow), chunked segmented sums with their partial
slots, the multi-level partial passes, the weighted reduction tree and the
Horner combine -- is replayed here with integers mod r standing in for group
elements (P_i -> p_i, phi(P) -> lambda*p).  Every index is checked against the
sizes the engine allocates from the same plan, every bucket must be written
at most once, and the result must equal sum s_i p_i mod r.  No GPU needed.
"""
import ctypes
import json
import random

import pytest

from oracle import pyref as R
from zkmetal_b200 import lib as zl


def plan(curve, counts, fmt=0, window=0, chunk=0, glv=-1, bits=0):
    L = zl.lib()
    arr = (ctypes.c_uint32 * len(counts))(*counts)
    buf = ctypes.create_string_buffer(1 << 22)
    st = L.zkmsm_plan_describe(curve, arr, len(counts), fmt, window, chunk, glv, bits, buf, len(buf))
    assert st == 0, zl.last_error()
    return json.loads(buf.value.decode())


def halves(C, s, glv):
    """Device prepare_scalar: integer mod r, then GLV split with signs."""
    s %= C.r
    if not glv:
        return [(s, 0)]
    k1, k2 = R.glv_split(C, s)
    return [(abs(k1), int(k1 < 0)), (abs(k2), int(k2 < 0))]


def win_width(c, nlo, w):
    return c + (1 if w >= nlo else 0)


def win_bit(c, nlo, w):
    return w * c + max(0, w - nlo)


def win_bucket(c, nlo, w):
    return (w + max(0, w - nlo)) << (c - 1)


def digits(k, c, nwin, nlo=None):
    """Signed digits; windows [0, nlo) are c bits, later ones c + 1 bits."""
    nlo = nwin if nlo is None else nlo
    carry = 0
    for w in range(nwin):
        cw = win_width(c, nlo, w)
        v = ((k >> win_bit(c, nlo, w)) & ((1 << cw) - 1)) + carry
        if v > (1 << (cw - 1)):
            yield w, (1 << cw) - v, 1
            carry = 1
        else:
            yield w, v, 0
            carry = 0


def excl_scan(a):
    out, run = [], 0
    for v in a:
        out.append(run)
        run += v
    return out, run


def plan_shift(curve, counts, shift_bits, table_points, window=0):
    L = zl.lib()
    arr = (ctypes.c_uint32 * len(counts))(*counts)
    buf = ctypes.create_string_buffer(1 << 22)
    st = L.zkmsm_plan_describe_shift(curve, arr, len(counts), 0, window, shift_bits, table_points, buf, len(buf))
    assert st == 0, zl.last_error()
    return json.loads(buf.value.decode())


def run_model(C, pl, bases, scalars, seed=0):
    """`bases`: the base table as the entries index it (for a shift-table
    plan, copy k of the table at k * table_points + i)."""
    r = C.r
    lam = C.lam
    rng = random.Random(seed)
    descs = pl["descs"]
    G = pl["nbuckets"]
    # 1-3: histogram, scan, scatter
    entries = []
    for d in descs:
        soff, n, boff, c, nwin, glv, bucket_off, fmt, win_off, wstep, nred, nlo = d
        for i in range(n):
            for j, (k, hneg) in enumerate(halves(C, scalars[soff + i], glv)):
                assert k < 1 << sum(win_width(c, nlo, w) for w in range(nwin)) - 1, "windows cover bits + 1"
                for w, a, dneg in digits(k, c, nwin, nlo):
                    if a:
                        if wstep:  # shift table: one bucket set, window w reads copy w*c/s
                            gb = bucket_off + (a - 1)
                            idx = boff + i + w * wstep
                            assert idx < len(bases) and idx <= 0x3FFFFFFF
                            entries.append((gb, idx | ((hneg ^ dneg) << 31)))
                        else:
                            gb = bucket_off + win_bucket(c, nlo, w) + (a - 1)
                            entries.append((gb, (boff + i) | (j << 30) | ((hneg ^ dneg) << 31)))
                        assert gb < G
    assert len(entries) <= pl["entry_bound"]
    rng.shuffle(entries)  # atomics give any order within a bucket
    entries.sort(key=lambda e: e[0])
    keys = [e[0] for e in entries]
    vals = [e[1] for e in entries]

    def point(v):
        idx = v & 0x3FFFFFFF
        x = bases[idx] * (lam if (v >> 30) & 1 else 1) % r
        return (-x) % r if v >> 31 else x

    buckets = [0] * G
    written = [False] * G

    def write_bucket(k, x):
        assert not written[k], "bucket %d written twice" % k
        written[k] = True
        buckets[k] = x % r

    cur_keys, cur_vals = keys, None
    M = len(keys)
    for lvl, (K, T, Mbound) in enumerate(pl["acc"]):
        assert M <= Mbound
        cnt = []
        for t in range(T):
            start = t * K
            if start >= M:
                cnt.append(0)
                continue
            end = min(start + K, M)
            k0, k1 = cur_keys[start], cur_keys[end - 1]
            cb = int(start > 0 and cur_keys[start - 1] == k0)
            ca = int(end < M and cur_keys[end] == k1)
            cnt.append((cb | ca) if k0 == k1 else cb + ca)
        pos, total = excl_scan(cnt)
        if lvl + 1 < len(pl["acc"]):
            assert total <= pl["acc"][lvl + 1][2], "partial slots exceed the next level's bound"
        else:
            assert total == 0, "last level must complete every bucket"
        pkeys = [None] * total
        pvals = [None] * total
        for t in range(T):
            start = t * K
            if start >= M:
                continue
            end = min(start + K, M)
            cur = cur_keys[start]
            cont_before = start > 0 and cur_keys[start - 1] == cur
            first_run = True
            slot = pos[t]
            acc = 0
            for i in range(start, end):
                k = cur_keys[i]
                if k != cur:
                    if first_run and cont_before:
                        pkeys[slot], pvals[slot] = cur, acc
                        slot += 1
                    else:
                        write_bucket(cur, acc)
                    acc, cur, first_run = 0, k, False
                acc += point(vals[i]) if lvl == 0 else cur_vals[i]
            cont_after = end < M and cur_keys[end] == cur
            if (first_run and cont_before) or cont_after:
                assert slot < total
                pkeys[slot], pvals[slot] = cur, acc
                slot += 1
            else:
                write_bucket(cur, acc)
            assert slot == pos[t] + cnt[t], "slot count disagrees with the chunk count pass"
        cur_keys, cur_vals, M = pkeys, pvals, total
    assert M == 0
    # bucket reduction tree
    L, log2L = pl["red_L"], pl["red_log2L"]
    inS, inW = buckets, None
    for lvl, tasks in enumerate(pl["red"]):
        nout = sum(t[3] for t in tasks)
        outS, outW = [None] * nout, [None] * nout
        for (in_off, n_in, out_off, n_out) in tasks:
            for local in range(n_out):
                g = out_off + local
                c0 = in_off + local * L
                cnt = min(L, n_in - local * L)
                run = x = 0
                for s in range(cnt - 1, 0, -1):
                    run += inS[c0 + s]
                    x += run
                run += inS[c0]
                outS[g] = run % r
                x = x * (1 << (lvl * log2L))
                if inW is not None:
                    x += sum(inW[c0 + s] for s in range(cnt))
                outW[g] = x % r
        inS, inW = outS, outW
    results = []
    for d in descs:
        soff, n, boff, c, nwin, glv, bucket_off, fmt, win_off, wstep, nred, nlo = d
        assert nred == (1 if wstep else nwin)
        acc = 0
        for w in range(nred - 1, -1, -1):
            acc = acc * (1 << win_width(c, nlo, w)) + inS[win_off + w] + inW[win_off + w]
        results.append(acc % r if n else 0)
    return results


CASES = [
    # curve, counts, dist, window, chunk, glv, bits
    ("bn254", [700], "uniform", 0, 0, -1, 0),
    ("bn254", [700], "witness", 0, 8, -1, 0),
    ("bn254", [2000], "witness", 6, 8, -1, 0),        # hot buckets -> several partial levels
    ("bn254", [300, 0, 17, 1, 900], "uniform", 0, 0, -1, 0),
    ("bn254", [500], "uniform", 11, 33, 0, 0),          # no GLV: 255-bit scalars
    ("bn254", [400], "uniform", 0, 0, -1, 16),          # small-scalar plan
    ("bls12_381", [600], "uniform", 16, 16, -1, 0),     # 9 windows for 128-bit halves
    ("bls12_381", [250, 0, 40], "witness", 0, 0, -1, 0),
    ("bls12_381", [300], "uniform", 13, 64, 0, 0),
    ("bls12_377", [500], "uniform", 0, 0, -1, 0),       # 126-bit GLV halves
    ("bls12_377", [200, 0, 33], "witness", 9, 16, 0, 0),
]


@pytest.mark.parametrize("curve,counts,dist,window,chunk,glv,bits", CASES)
def test_schedule_model(curve, counts, dist, window, chunk, glv, bits):
    C = R.CURVES[curve]
    cid = {"bn254": zl.BN254, "bls12_381": zl.BLS12_381, "bls12_377": zl.BLS12_377}[curve]
    pl = plan(cid, counts, 0, window, chunk, glv, bits)
    rng = random.Random(sum(counts) + window)
    total = sum(counts)
    bases = [rng.randrange(1, C.r) for _ in range(total)]
    if bits:
        scalars = [rng.getrandbits(bits) for _ in range(total)]
    elif dist == "uniform":
        scalars = [rng.randrange(1 << 256) for _ in range(total)]
    else:
        scalars = []
        for _ in range(total):
            u = rng.randrange(100)
            scalars.append(0 if u < 40 else 1 if u < 60 else rng.getrandbits(32) if u < 85 else rng.randrange(C.r))
    got = run_model(C, pl, bases, scalars, seed=len(counts))
    off = 0
    for m, n in enumerate(counts):
        # the plan puts every MSM on a prefix of one base table (base_off = 0)
        want = sum(s * b for s, b in zip(scalars[off:off + n], bases[:n])) % C.r
        assert got[m] == want, m
        off += n


LAYOUT_CASES = [
    # curve, counts, dist, c, nlo (nlo windows of c bits, then c + 1-bit ones)
    ("bn254", [700], "uniform", 5, 10),
    ("bn254", [2000], "witness", 6, 1),
    ("bn254", [300, 0, 17, 1, 900], "uniform", 7, 4),
    ("bls12_381", [600], "uniform", 8, 3),
    ("bls12_381", [250, 0, 40], "witness", 4, 20),
]


@pytest.mark.parametrize("curve,counts,dist,c,nlo", LAYOUT_CASES)
def test_schedule_model_two_width(curve, counts, dist, c, nlo):
    """Forced two-width layouts (window setting c | nlo << 16): digits,
    bucket offsets, reduction tasks and the Horner combine per window width."""
    C = R.CURVES[curve]
    cid = zl.BN254 if curve == "bn254" else zl.BLS12_381
    pl = plan(cid, counts, 0, c | (nlo << 16), 0, -1, 0)
    for d in pl["descs"]:
        if d[1]:
            assert d[3] == c and d[11] == nlo < d[4]
    rng = random.Random(sum(counts) + c)
    total = sum(counts)
    bases = [rng.randrange(1, C.r) for _ in range(total)]
    if dist == "uniform":
        scalars = [rng.randrange(1 << 256) for _ in range(total)]
    else:
        scalars = [0 if u < 40 else 1 if u < 60 else rng.getrandbits(32) if u < 85 else rng.randrange(C.r)
                   for u in (rng.randrange(100) for _ in range(total))]
    got = run_model(C, pl, bases, scalars, seed=len(counts))
    off = 0
    for m, n in enumerate(counts):
        want = sum(sc * b for sc, b in zip(scalars[off:off + n], bases[:n])) % C.r
        assert got[m] == want, m
        off += n


SHIFT_CASES = [
    # curve, counts, dist, shift spacing, table points, window override
    ("bn254", [700], "uniform", 4, 700, 0),
    ("bn254", [700], "witness", 4, 1000, 0),
    ("bn254", [300, 0, 17, 1, 900], "uniform", 4, 1000, 0),
    ("bn254", [500], "uniform", 4, 600, 10),   # 10 rounds up to a multiple of 4
    ("bn254", [400], "witness", 8, 400, 16),
    ("bls12_381", [600], "uniform", 6, 600, 0),
    ("bls12_381", [250, 0, 40], "witness", 5, 300, 0),
]


@pytest.mark.parametrize("curve,counts,dist,s,tp,window", SHIFT_CASES)
def test_schedule_model_shift_table(curve, counts, dist, s, tp, window):
    """MSMs over a table with window shifts: every window's digits index
    copy w*c/s of the table and add into one bucket set; one window sum."""
    C = R.CURVES[curve]
    cid = zl.BN254 if curve == "bn254" else zl.BLS12_381
    pl = plan_shift(cid, counts, s, tp, window)
    for d in pl["descs"]:
        if d[1]:
            assert d[3] % s == 0 and d[5] == 0 and d[10] == 1 and d[9] == (d[3] // s) * tp
            if window:
                assert d[3] == -(-window // s) * s
    copies = -(-(C.r.bit_length() + 1) // s)
    rng = random.Random(sum(counts) + s)
    table = [rng.randrange(1, C.r) for _ in range(tp)]
    ext = [p * pow(2, s * k, C.r) % C.r for k in range(copies) for p in table]
    total = sum(counts)
    if dist == "uniform":
        scalars = [rng.randrange(1 << 256) for _ in range(total)]
    else:
        scalars = []
        for _ in range(total):
            u = rng.randrange(100)
            scalars.append(0 if u < 40 else 1 if u < 60 else rng.getrandbits(32) if u < 85 else rng.randrange(C.r))
    got = run_model(C, pl, ext, scalars, seed=len(counts))
    off = 0
    for m, n in enumerate(counts):
        want = sum(sc * b for sc, b in zip(scalars[off:off + n], table[:n])) % C.r
        assert got[m] == want, m
        off += n


def test_shift_plan_falls_back_outside_table():
    """An MSM longer than the shift table's prefix uses ordinary windows."""
    pl = plan_shift(zl.BN254, [100, 5000], 4, 1000)
    assert pl["descs"][0][9] > 0 and pl["descs"][0][10] == 1
    assert pl["descs"][1][9] == 0 and pl["descs"][1][10] == pl["descs"][1][4]


def test_plan_sizes_2_24():
    """The full-size plan: entry and bucket counts fit 32-bit indices and the
    window choice is the cost model's."""
    pl = plan(zl.BN254, [1 << 24])
    d = pl["descs"][0]
    c, nwin, nlo = d[3], d[4], d[11]
    assert win_bucket(c, nlo, nwin) == pl["nbuckets"]
    assert pl["entry_bound"] == 2 * (1 << 24) * nwin < (1 << 32)
    assert 14 <= c <= 22
    # GLV halves of 127 bits: the windows cover exactly the 128 bits of the
    # signed recoding, the wider ones on top
    assert sum(win_width(c, nlo, w) for w in range(nwin)) == 128 and nlo <= nwin


@pytest.mark.parametrize("curve,n", [("bn254", 1 << 20), ("bn254", 1 << 22), ("bn254", 1 << 24),
                                     ("bls12_381", 1 << 22)])
def test_two_width_layout_covers_scalar(curve, n):
    """Large plans split the signed recoding's bits + 1 bits into windows
    whose widths differ by at most one."""
    cid = zl.BN254 if curve == "bn254" else zl.BLS12_381
    d = plan(cid, [n])["descs"][0]
    c, nwin, nlo = d[3], d[4], d[11]
    widths = [win_width(c, nlo, w) for w in range(nwin)]
    assert max(widths) - min(widths) <= 1 and widths == sorted(widths)
    assert sum(widths) - widths[-1] < 128 <= sum(widths)


def _types_const(name):
    import os
    import re
    text = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "zkmetal_b200", "csrc",
                             "types.cuh")).read()
    m = re.search(r"constexpr\s+\w+\s+%s\s*=\s*([^;]+);" % name, text)
    return int(m.group(1))


@pytest.mark.parametrize("curve,counts,window,glv", [
    (0, [1 << 24], 0, -1), (0, [1 << 20], 0, -1), (0, [1 << 12], 0, -1), (0, [3000], 6, -1), (0, [5000], 2, 0),
    (1, [1 << 22], 0, -1), (2, [1 << 16], 0, -1), (3, [1 << 14], 0, -1), (0, [4096, 1 << 20, 333, 1 << 18], 0, -1),
    (0, [1 << 10] * 64, 0, 0), (0, [100], 3 | 1 << 16, -1)])
def test_digit_block_slices_fit(curve, counts, window, glv):
    """k_radix_digits gives each warp a slice of SORT_DBUF / 8 entries and runs
    min(32, spb / 8) lanes per warp in rounds of 8 * lanes scalars: for the
    plan's scalars per block (spb) and digits per scalar (maxd), a warp's
    digits of all its rounds must fit its slice."""
    dbuf, threads = _types_const("SORT_DBUF"), _types_const("SORT_DTHREADS")
    warps = threads // 32
    pl = plan(curve, counts, window=window, glv=glv)
    maxd, spb = pl["sort"][0], pl["sort"][1]
    assert maxd >= 1 and spb >= warps
    lanes = min(32, spb // warps)
    rounds = -(-spb // (warps * lanes))
    assert lanes >= 1 and rounds * lanes * maxd <= dbuf // warps, (maxd, spb, lanes, rounds)
    # the same number of scalars per block as the kernel's rounds cover
    assert spb <= rounds * warps * lanes
