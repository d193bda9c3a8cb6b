"""Parity of the CUDA MSM with the oracle, through the C ABI (GPU required).

Shapes follow the reference tests (Tests/zkMetalTests/MSMTests.swift:7-108:
5*G, n = 1..64 against a naive sum, scalar 0 / 1, determinism across runs
and engines, on-curve; DASTests.swift:8-150: the BLS12-381 469*G answers),
plus what the reference never checks on its GPU path: large n against the
compiled reference C Pippenger, skewed (witness-like) scalars, duplicate and
cancelling bases, identity bases, unreduced and maximal scalars, every
tuning knob giving the same result, and the batch entry points.
Bar: bit-exact affine results."""
import ctypes
import json
import os
import random

import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import (CURVE_ID, check, gen_inputs, jac_to_affine_bytes, msm_device, np_bytes, oracle_msm,
                               to_host)
from zkmetal_b200 import BLS12377MSM, BLS12381MSM, CommitmentTable, MetalMSM, MSMError, multiMSM
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "msm_golden.json")
ENGINES = {"bn254": MetalMSM, "bls12_381": BLS12381MSM, "bls12_377": BLS12377MSM}
CURVES3 = ["bn254", "bls12_381", "bls12_377"]
# drop-in host entry points per curve: integer scalars, Montgomery scalars, batch
FR_FN = {"bn254": "zkmetal_bn254_msm_fr", "bls12_381": "zkmetal_bls12_381_g1_msm_fr",
         "bls12_377": "zkmetal_bls12_377_g1_msm_fr"}
BATCH_FN = {"bn254": "zkmetal_bn254_msm_batch", "bls12_381": "zkmetal_bls12_381_g1_msm_batch",
            "bls12_377": "zkmetal_bls12_377_g1_msm_batch"}


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return {"bn254": MetalMSM(), "bls12_381": BLS12381MSM(), "bls12_377": BLS12377MSM()}


def aff(C, res):
    return jac_to_affine_bytes(C, res.x + res.y + res.z)


def test_gpu_available(eng):
    assert zl.lib().zkmetal_gpu_available() == 1


@pytest.mark.parametrize("curve", CURVES3)
def test_5G(eng, curve):
    C = R.CURVES[curve]
    G = (C.gx, C.gy)
    r = eng[curve].msm(C.enc_affine(G), R.pack_scalars_int([5]))
    assert aff(C, r) == C.enc_affine(R.scalar_mul(C, G, 5))


with open(GOLDEN) as _f:
    _G = json.load(_f)


@pytest.mark.parametrize("case", _G["cases"], ids=lambda c: "%s-%d-%d-%s" % (c["curve"], c["seed"], c["n"], c["dist"]))
def test_golden_cases(eng, case):
    C = R.CURVES[case["curve"]]
    pts = R.make_bases(C, case["seed"], case["n"])
    sc = R.make_scalars(C, case["seed"], case["n"], case["dist"])
    want = bytes.fromhex(case["result_affine"])
    e = eng[case["curve"]]
    assert aff(C, e.msm(R.pack_points(C, pts), R.pack_scalars_int(sc))) == want
    assert aff(C, e.msmFr(R.pack_points(C, pts), R.pack_scalars_mont(C, sc))) == want


@pytest.mark.parametrize("kat", _G["kat"], ids=lambda k: "%s-%s" % (k["curve"], k["name"]))
def test_golden_kats(eng, kat):
    C = R.CURVES[kat["curve"]]
    pb = b"".join(bytes.fromhex(p) for p in kat["points"])
    r = eng[kat["curve"]].msm(pb, R.pack_scalars_int(kat["scalars"]))
    assert aff(C, r) == bytes.fromhex(kat["result_affine"])


@pytest.mark.parametrize("curve", CURVES3)
def test_prefixes_vs_naive(eng, curve):
    """MSMTests.swift:56-62 shape: n in {1, 2, 4, ..., 64} against naive sums."""
    C = R.CURVES[curve]
    pts = R.make_bases(C, 31, 64)
    sc = [random.Random(31).getrandbits(256) for _ in range(64)]
    for n in (1, 2, 4, 8, 16, 32, 64):
        want = C.enc_affine(R.naive_msm(C, pts[:n], sc[:n]))
        assert aff(C, eng[curve].msm(R.pack_points(C, pts[:n]), R.pack_scalars_int(sc[:n]))) == want, n


@pytest.mark.parametrize("curve", CURVES3)
def test_edge_cases(eng, curve):
    C = R.CURVES[curve]
    G = (C.gx, C.gy)
    P = R.scalar_mul(C, G, 987654321)
    Q = R.aff_neg(C, P)
    cases = [
        ([P, P, P], [3, 3, 3]),                         # duplicate bases in one bucket (doubling path)
        ([P, Q], [9, 9]),                               # cancel to the identity
        ([P, Q, P], [9, 9, 2]),
        ([None, P, None], [5, 7, 11]),                  # identity bases (0, 0)
        ([P, G], [0, 0]),                               # all-zero scalars
        ([P, G], [1, 1]),
        ([P, G, P], [C.r - 1, C.r, C.r + 5]),           # unreduced integer scalars
        ([P, G], [(1 << 256) - 1, (1 << 255)]),
        ([G] * 40, [1] * 40),                           # one hot bucket
    ]
    L = zl.lib()
    try:
        # default plan, a two-width layout (c | nlo << 16), and no GLV
        for window, glv in ((0, -1), (5 | 10 << 16, 1), (6 | 3 << 16, 0)):
            check(L.zkmsm_engine_set_tuning(eng[curve].handle, window, 0, glv))
            for pts, sc in cases:
                want = C.enc_affine(R.naive_msm(C, pts, sc))
                got = aff(C, eng[curve].msm(R.pack_points(C, pts), R.pack_scalars_int(sc)))
                assert got == want, (window, glv, pts, sc)
    finally:
        check(L.zkmsm_engine_set_tuning(eng[curve].handle, 0, 0, -1))


def glv_boundary_scalars(C):
    """Scalars where the GLV split is most fragile: within one of a Babai
    rounding boundary s*G_j / 2^256 = k + 1/2 (c_j flips there), around
    lambda and its multiples, the extremes of [0, r) and the half-width
    powers of two."""
    g = C.glv
    out = set()
    for gj in (g["g1"], g["g2"]):
        top = (C.r * gj) >> 256
        for k in [0, 1, 2, 3, 1000, top // 3, top // 2, top - 2, top - 1, top]:
            for d in (-1, 0, 1):
                s = (((2 * k + 1) << 255) // gj) + d
                if 0 <= s < C.r:
                    out.add(s)
    for s in (0, 1, 2, C.lam - 1, C.lam, C.lam + 1, 2 * C.lam % C.r, C.r - C.lam, C.r - 1, C.r - 2,
              (C.r - 1) // 2, (C.r + 1) // 2, (1 << 127) - 1, 1 << 127, (1 << 128) - 1, 1 << 128):
        out.add(s % C.r)
    return sorted(out)


@pytest.mark.parametrize("curve", CURVES3)
def test_glv_rounding_boundaries(eng, curve):
    """Every boundary scalar of the GLV split, as integer and as Montgomery
    input, against the naive sum (one MSM of all of them, and each alone so
    that one wrong split cannot hide behind another)."""
    C = R.CURVES[curve]
    e = eng[curve]
    sc = glv_boundary_scalars(C)
    pts = R.make_bases(C, 77, len(sc))
    want = C.enc_affine(R.naive_msm(C, pts, sc))
    assert aff(C, e.msm(R.pack_points(C, pts), R.pack_scalars_int(sc))) == want
    assert aff(C, e.msmFr(R.pack_points(C, pts), R.pack_scalars_mont(C, sc))) == want
    G = (C.gx, C.gy)
    for s in sc:
        one = C.enc_affine(R.naive_msm(C, [G], [s]))
        assert aff(C, e.msmFr(R.pack_points(C, [G]), R.pack_scalars_mont(C, [s]))) == one, hex(s)


def test_invalid_inputs(eng):
    e = eng["bn254"]
    with pytest.raises(MSMError) as ei:
        e.msm(b"", b"")
    assert ei.value.case == "invalidInput"
    with pytest.raises(MSMError):
        e.msm(bytes(64 * 2), bytes(32))
    buf = ctypes.create_string_buffer(96)
    assert zl.lib().zkmetal_bn254_msm(e.handle, buf, buf, 0, buf, buf, buf) == zl.ERR_INVALID_INPUT
    assert zl.lib().zkmetal_bn254_msm_batch(e.handle, buf, buf, buf, 0, buf) == zl.ERR_INVALID_INPUT


@pytest.mark.parametrize("curve", CURVES3)
def test_generator_matches_restatement(eng, curve):
    C = R.CURVES[curve]
    n = 12
    for dist in ("uniform", "witness"):
        for fmt in (zl.SCALAR_INT, zl.SCALAR_MONT):
            p, s = gen_inputs(eng[curve], curve, 5, n, dist, fmt)
            assert to_host(p) == R.pack_points(C, R.make_bases(C, 5, n))
            sc = R.make_scalars(C, 5, n, dist)
            want = R.pack_scalars_mont(C, sc) if fmt == zl.SCALAR_MONT else R.pack_scalars_int(sc)
            assert to_host(s) == want


@pytest.mark.parametrize("curve,n,dist", [("bn254", 4096, "uniform"), ("bn254", 4096, "witness"),
                                          ("bn254", 1 << 16, "uniform"), ("bn254", 1 << 16, "witness"),
                                          ("bls12_381", 4096, "uniform"), ("bls12_381", 1 << 16, "witness"),
                                          ("bls12_381", 1 << 16, "uniform"), ("bls12_377", 4096, "uniform"),
                                          ("bls12_377", 4096, "witness"), ("bls12_377", 1 << 16, "uniform")])
def test_vs_reference_c(eng, oracles, curve, n, dist):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    p, s = gen_inputs(eng[curve], curve, 100 + n, n, dist, zl.SCALAR_MONT)
    got = jac_to_affine_bytes(C, msm_device(eng[curve], curve, p, s, zl.SCALAR_MONT, n))
    want = oracle_msm(orc, curve, to_host(p), to_host(s), n, zl.SCALAR_MONT)
    assert got == want


@pytest.mark.parametrize("curve", CURVES3)
def test_tuning_invariance(eng, oracles, curve):
    """Window width, chunk length and GLV on/off change the schedule, never the result."""
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    n = 3000
    p, s = gen_inputs(eng[curve], curve, 77, n, "witness", zl.SCALAR_INT)
    e = eng[curve]
    L = zl.lib()
    results = set()
    try:
        # c | nlo << 16: nlo windows of c bits, then c + 1-bit windows
        for c, k, glv in [(0, 0, -1), (6, 8, 1), (11, 33, 1), (16, 128, 1), (21, 16, 1), (9, 8, 0), (13, 64, 0),
                          (5 | 10 << 16, 8, 1), (12 | 3 << 16, 16, 1), (18 | 5 << 16, 64, 1), (21 | 4 << 16, 192, 1),
                          (10 | 7 << 16, 24, 0)]:
            check(L.zkmsm_engine_set_tuning(e.handle, c, k, glv))
            results.add(msm_device(e, curve, p, s, zl.SCALAR_INT, n))
    finally:
        check(L.zkmsm_engine_set_tuning(e.handle, 0, 0, -1))
    assert len(results) == 1
    assert jac_to_affine_bytes(C, results.pop()) == oracle_msm(orc, curve, to_host(p), to_host(s), n, zl.SCALAR_INT)


@pytest.mark.parametrize("curve", CURVES3)
def test_determinism_across_runs_and_engines(eng, curve):
    C = R.CURVES[curve]
    n = 32768
    p, s = gen_inputs(eng[curve], curve, 9, n, "uniform", zl.SCALAR_MONT)
    r1 = msm_device(eng[curve], curve, p, s, zl.SCALAR_MONT, n)
    r2 = msm_device(eng[curve], curve, p, s, zl.SCALAR_MONT, n)
    other = ENGINES[curve]()
    r3 = msm_device(other, curve, p, s, zl.SCALAR_MONT, n)
    other.close()
    assert r1 == r2 == r3
    assert C.on_curve(C.dec_affine(jac_to_affine_bytes(C, r1)))


def test_small_scalar_variants(eng):
    C = R.BN254
    e = eng["bn254"]
    L = zl.lib()
    n = 200
    pts = R.make_bases(C, 41, n)
    pb = np_bytes(R.pack_points(C, pts))
    rng = random.Random(41)
    for width, fn in ((1, L.zkmetal_bn254_msm_u8), (2, L.zkmetal_bn254_msm_u16), (4, L.zkmetal_bn254_msm_u32)):
        sc = [rng.getrandbits(8 * width) for _ in range(n)]
        sb = np_bytes(b"".join(v.to_bytes(width, "little") for v in sc))
        rx, ry, rz = (ctypes.create_string_buffer(32) for _ in range(3))
        check(fn(e.handle, pb.ctypes.data, sb.ctypes.data, n, rx, ry, rz))
        assert jac_to_affine_bytes(C, rx.raw + ry.raw + rz.raw) == C.enc_affine(R.naive_msm(C, pts, sc))


@pytest.mark.parametrize("curve", CURVES3)
@pytest.mark.parametrize("dist", ["uniform", "witness"])
def test_striped_host_msm_matches_unstriped(eng, oracles, curve, dist):
    """Host-buffer MSMs streamed in stripes (consecutive point ranges, the
    copy of stripe s overlapping the work on stripe s-1, one bucket array per
    stripe, the arrays added and reduced once) give the same point as the
    unstriped MSM and as the oracle; n is no multiple of the stripe, so the
    last stripe is shorter."""
    C = R.CURVES[curve]
    E = ENGINES[curve]()
    L = zl.lib()
    n = 3 * 4096 + 777
    p, s = gen_inputs(E, curve, 901, n, dist, zl.SCALAR_MONT)
    pb = np.frombuffer(to_host(p), dtype=np.uint8).copy()
    sb = np.frombuffer(to_host(s), dtype=np.uint8).copy()
    fn = getattr(L, FR_FN[curve])
    outs = []
    for stripe_log2 in (0, 12, 11, 13):
        check(L.zkmsm_engine_set_stripe(E.handle, stripe_log2))
        rx, ry, rz = (ctypes.create_string_buffer(C.fp_bytes) for _ in range(3))
        check(fn(E.handle, pb.ctypes.data, sb.ctypes.data, n, rx, ry, rz))
        outs.append(rx.raw + ry.raw + rz.raw)
    assert outs[0] == outs[1] == outs[2] == outs[3]
    ref, cm = oracles
    orc = ref if ref is not None else cm
    assert jac_to_affine_bytes(C, outs[0]) == oracle_msm(orc, curve, pb.tobytes(), sb.tobytes(), n, zl.SCALAR_MONT)
    assert L.zkmsm_engine_set_stripe(E.handle, 40) == zl.ERR_INVALID_INPUT
    assert L.zkmsm_engine_set_stripe(E.handle, -2) == zl.ERR_INVALID_INPUT
    check(L.zkmsm_engine_set_stripe(E.handle, -1))
    E.close()


@pytest.mark.parametrize("curve", CURVES3)
def test_batch_entry_point_matches_plain(eng, curve):
    """zkmetal_*_msm_batch: concatenated inputs, count 0 -> 96/144 zero bytes
    (zkMetal_ffi.swift:1260-1264); each result equals its own plain call."""
    C = R.CURVES[curve]
    e = eng[curve]
    counts = [5, 0, 300, 1, 64]
    total = sum(counts)
    pts = R.make_bases(C, 51, total)
    sc = R.make_scalars(C, 51, total, "witness")
    pb, sb = np_bytes(R.pack_points(C, pts)), np_bytes(R.pack_scalars_int(sc))
    cnt = np.array(counts, dtype=np.uint32)
    out = ctypes.create_string_buffer(len(counts) * 3 * C.fp_bytes)
    fn = getattr(zl.lib(), BATCH_FN[curve])
    check(fn(e.handle, pb.ctypes.data, sb.ctypes.data, cnt.ctypes.data, len(counts), out))
    f3 = 3 * C.fp_bytes
    off = 0
    for i, c in enumerate(counts):
        got = out.raw[i * f3:(i + 1) * f3]
        if c == 0:
            assert got == bytes(f3)
        else:
            plain = e.msm(R.pack_points(C, pts[off:off + c]), R.pack_scalars_int(sc[off:off + c]))
            assert got == plain.x + plain.y + plain.z
            assert jac_to_affine_bytes(C, got) == C.enc_affine(R.naive_msm(C, pts[off:off + c], sc[off:off + c]))
        off += c


@pytest.mark.parametrize("curve", CURVES3)
def test_resident_table_batch_commit(eng, curve):
    """Many uneven MSMs over prefixes of one resident table, bit-exact against
    separate plain calls (the batched-commitments pattern)."""
    C = R.CURVES[curve]
    e = eng[curve]
    T = 1 << 14
    p, _ = gen_inputs(e, curve, 61, T, "uniform", zl.SCALAR_MONT)
    rng = random.Random(61)
    counts = [int(2 ** rng.uniform(4, 14)) for _ in range(9)] + [T, 1, 0]
    _, s = gen_inputs(e, curve, 62, sum(counts), "uniform", zl.SCALAR_MONT)
    table = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        res = table.batch_commit(s.data_ptr(), counts, fmt=zl.SCALAR_MONT, on_device=True)
        res2 = table.batch_commit(s.data_ptr(), counts, fmt=zl.SCALAR_MONT, on_device=True)
    finally:
        table.close()
    off = 0
    for i, c in enumerate(counts):
        got = res[i].x + res[i].y + res[i].z
        assert got == res2[i].x + res2[i].y + res2[i].z
        if c == 0:
            assert got == bytes(3 * C.fp_bytes)
        else:
            sub = s[off * 32:(off + c) * 32]
            assert got == msm_device(e, curve, p, sub, zl.SCALAR_MONT, c), i
        off += c


def test_multi_msm_matches_single(eng):
    C = R.BN254
    e = eng["bn254"]
    n = 100
    pts = R.make_bases(C, 71, n)
    sets = [R.make_scalars(C, 71 + k, n, "uniform") for k in range(3)]
    res = multiMSM(e, R.pack_points(C, pts), [R.pack_scalars_int(s) for s in sets])
    for r, s in zip(res, sets):
        single = e.msm(R.pack_points(C, pts), R.pack_scalars_int(s))
        assert (r.x, r.y, r.z) == (single.x, single.y, single.z)


@pytest.mark.slow
@pytest.mark.parametrize("curve,dist", [("bn254", "uniform"), ("bn254", "witness"), ("bls12_381", "uniform"),
                                        ("bls12_377", "uniform")])
def test_2_20_vs_reference_c(eng, oracles, curve, dist):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    n = 1 << 20
    p, s = gen_inputs(eng[curve], curve, 2020, n, dist, zl.SCALAR_MONT)
    got = jac_to_affine_bytes(C, msm_device(eng[curve], curve, p, s, zl.SCALAR_MONT, n))
    assert got == oracle_msm(orc, curve, to_host(p), to_host(s), n, zl.SCALAR_MONT)


@pytest.mark.slow
@pytest.mark.parametrize("dist", ["uniform", "witness"])
def test_2_24_split_linearity(eng, oracles, dist):
    """Full-size property check: MSM over 2^24 points equals the sum of the
    MSMs over its two halves (different window widths are chosen for n and
    n/2, so the two sides follow different schedules)."""
    _, cm = oracles
    C = R.BN254
    n = 1 << 24
    e = eng["bn254"]
    p, s = gen_inputs(e, "bn254", 2424, n, dist, zl.SCALAR_MONT)
    full = jac_to_affine_bytes(C, msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n))
    h = n // 2
    a = jac_to_affine_bytes(C, msm_device(e, "bn254", p[:h * 64], s[:h * 32], zl.SCALAR_MONT, h))
    b = jac_to_affine_bytes(C, msm_device(e, "bn254", p[h * 64:], s[h * 32:], zl.SCALAR_MONT, h))
    assert full == cm.affine_add("bn254", a, b)
    assert C.on_curve(C.dec_affine(full))


def test_small_dropin_graph_sequence():
    """Drop-in calls of up to 2^16 points run their launches directly on the
    first call of a size, capture a CUDA graph on the second and replay it
    after that.  Every call must equal the device-pointer MSM of the same
    inputs: with new scalars between replays, other sizes interleaved, and a
    larger call that regrows the workspace and drops the captured graphs."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = MetalMSM()  # fresh engine: no plans or graphs yet
    try:
        N = 1 << 13
        p, s1 = gen_inputs(e, "bn254", 501, N, "uniform", zl.SCALAR_MONT)
        _, s2 = gen_inputs(e, "bn254", 502, N, "witness", zl.SCALAR_MONT)
        ph = to_host(p)
        sh = {1: to_host(s1), 2: to_host(s2)}
        sd = {1: s1, 2: s2}
        seq = [(1000, 1), (1000, 1), (1000, 2), (1000, 1), (777, 2), (1000, 2), (N, 1), (1000, 1), (1000, 2),
               (1000, 1), (777, 1), (777, 2)]
        for n, k in seq:
            r = e.msmFr(ph[:n * 64], sh[k][:n * 32])
            assert r.x + r.y + r.z == msm_device(e, "bn254", p, sd[k], zl.SCALAR_MONT, n), (n, k)
    finally:
        e.close()


@pytest.mark.parametrize("curve,n", [("bn254", (1 << 17) + 5), ("bn254", 1 << 20), ("bn254", 1 << 21),
                                     ("bls12_381", 1 << 20)])
def test_dropin_pinned_buffers_overlap(eng, curve, n):
    """Drop-in calls from pinned host buffers, where the copies really run
    under the computation: above 2^16 points the bases arrive on a second
    stream while the scalars are sorted, and from 2^21 BN254 points each
    stripe's sort waits only for its scalars.  Each call must equal the
    device-pointer MSM of the same inputs, also when the host buffers are
    refilled between calls."""
    e = eng[curve]
    C = R.CURVES[curve]
    fn = {"bn254": zl.lib().zkmetal_bn254_msm_fr, "bls12_381": zl.lib().zkmetal_bls12_381_g1_msm_fr}[curve]
    rx, ry, rz = (ctypes.create_string_buffer(C.fp_bytes) for _ in range(3))
    ph = torch.empty(n * 2 * C.fp_bytes, dtype=torch.uint8).pin_memory()
    sh = torch.empty(n * 32, dtype=torch.uint8).pin_memory()
    for seed in (701, 702, 703):
        p, s = gen_inputs(e, curve, seed, n, "uniform" if seed != 702 else "witness", zl.SCALAR_MONT)
        ph.copy_(p.cpu())
        sh.copy_(s.cpu())
        check(fn(e.handle, ph.data_ptr(), sh.data_ptr(), n, rx, ry, rz))
        assert rx.raw + ry.raw + rz.raw == msm_device(e, curve, p, s, zl.SCALAR_MONT, n), seed


@pytest.mark.parametrize("dist", ["uniform", "witness"])
def test_sampled_layout_same_result(eng, dist):
    """The window layout chosen from a sample of the scalars (on by default
    from 2^21 points) changes the schedule, never the result: device calls
    (synchronous and on a stream) and a drop-in host call with sampling on
    equal the call with sampling off."""
    e = eng["bn254"]
    n = (1 << 21) + 123
    p, s = gen_inputs(e, "bn254", 881, n, dist, zl.SCALAR_MONT)
    L = zl.lib()
    check(L.zkmsm_engine_set_sampling(e.handle, 0))
    want = msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n)
    check(L.zkmsm_engine_set_sampling(e.handle, 1))
    assert msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n) == want
    out = torch.zeros(96, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    check(L.zkmsm_msm_device_async(e.handle, 0, p.data_ptr(), None, s.data_ptr(), zl.SCALAR_MONT, n, out.data_ptr(),
                                   ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    assert out.cpu().numpy().tobytes() == want
    r = e.msmFr(to_host(p), to_host(s))
    assert r.x + r.y + r.z == want


@pytest.mark.parametrize("curve,n", [("bn254", (1 << 20) + 9), ("bn254", (1 << 21) + 3), ("bls12_381", 1 << 20)])
def test_dropin_pageable_buffers_staged(eng, curve, n):
    """Drop-in calls from pageable host arrays (what a Swift [PointAffine] or a
    numpy array hands over): copies of 8 MB and more go through the engine's
    pinned staging ring, filled by host threads chunk by chunk while earlier
    chunks are on the bus.  Each call, unstriped and striped, equals the
    device-pointer MSM, also when the arrays are refilled between calls."""
    e = eng[curve]
    C = R.CURVES[curve]
    fn = {"bn254": zl.lib().zkmetal_bn254_msm_fr, "bls12_381": zl.lib().zkmetal_bls12_381_g1_msm_fr}[curve]
    rx, ry, rz = (ctypes.create_string_buffer(C.fp_bytes) for _ in range(3))
    ph = np.empty(n * 2 * C.fp_bytes, dtype=np.uint8)
    sh = np.empty(n * 32, dtype=np.uint8)
    for seed in (711, 712):
        p, s = gen_inputs(e, curve, seed, n, "uniform" if seed == 711 else "witness", zl.SCALAR_MONT)
        ph[:] = p.cpu().numpy()
        sh[:] = s.cpu().numpy()
        check(fn(e.handle, ph.ctypes.data, sh.ctypes.data, n, rx, ry, rz))
        assert rx.raw + ry.raw + rz.raw == msm_device(e, curve, p, s, zl.SCALAR_MONT, n), seed
