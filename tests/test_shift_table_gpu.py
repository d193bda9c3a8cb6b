"""Shift tables: fixed-base precomputation over a resident base table (GPU).

zkmsm_table_precompute extends a table with its window shifts (copy k of
point i = 2^(s*k) * P_i).  The copies must equal the oracle's scalar
multiples, and batched commitments and served requests over the table must
equal, bit for bit, the plain MSM of the same scalars over the same prefix
(and the oracle on small cases), for every spacing and scalar form.
"""
import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import check, gen_inputs, jac_to_affine_bytes, msm_device, oracle_msm, to_host
from zkmetal_b200 import BLS12377MSM, BLS12381MSM, CommitmentServer, CommitmentTable, MetalMSM, MSMError
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return {"bn254": MetalMSM(), "bls12_381": BLS12381MSM(), "bls12_377": BLS12377MSM()}


def table_bytes(table, nbytes):
    out = np.zeros(nbytes, dtype=np.uint8)
    check(zl.lib().zkmsm_memcpy_d2h(out.ctypes.data, zl.lib().zkmsm_table_device_points(table._h), nbytes))
    return out.tobytes()


def host_scalars(e, curve, seed, n, dist, fmt):
    _, s = gen_inputs(e, curve, seed, n, dist, fmt)
    return np.frombuffer(to_host(s), dtype=np.uint8).copy()


def plain(e, curve, d_points, scal_np, fmt, n):
    s = torch.from_numpy(scal_np[: n * 32].copy()).cuda()
    return msm_device(e, curve, d_points, s, fmt, n)


@pytest.mark.parametrize("curve,spacing", [("bn254", 4), ("bls12_381", 5)])
def test_shift_copies_are_window_shifts(eng, oracles, curve, spacing):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    e = eng[curve]
    n = 300
    p, _ = gen_inputs(e, curve, 41, n, "uniform", zl.SCALAR_MONT)
    p[7 * 2 * C.fp_bytes:8 * 2 * C.fp_bytes] = 0  # one identity point (0, 0)
    t = CommitmentTable(e, p.data_ptr(), on_device=True, n=n)
    try:
        t.precompute(spacing)
        assert t.shift_bits == spacing
        copies = -(-(C.r.bit_length() + 1) // spacing)
        ab = 2 * C.fp_bytes
        raw = table_bytes(t, copies * n * ab)
        pts = to_host(p)
        assert raw[:n * ab] == pts[:n * ab], "copy 0 is the table itself"
        for k in (1, 2, copies // 2, copies - 1):
            scal = (1 << (spacing * k)).to_bytes(32, "little")
            for i in (0, 7, 123, n - 1):
                got = raw[(k * n + i) * ab:(k * n + i + 1) * ab]
                if i == 7:
                    assert got == bytes(ab)
                else:
                    assert got == orc.msm(curve, pts[i * ab:(i + 1) * ab], scal, 1), (k, i)
    finally:
        t.close()


@pytest.mark.parametrize("curve,spacing,T", [("bn254", 4, 1 << 13), ("bn254", 6, 1 << 12),
                                             ("bls12_381", 4, 1 << 12), ("bls12_377", 5, 1 << 12)])
@pytest.mark.parametrize("dist,fmt", [("uniform", zl.SCALAR_MONT), ("witness", zl.SCALAR_INT)])
def test_shift_batch_matches_plain(eng, curve, spacing, T, dist, fmt):
    e = eng[curve]
    p, _ = gen_inputs(e, curve, 52, T, "uniform", zl.SCALAR_MONT)
    t = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        counts = [1, 2, 100, T // 2, 0, 777, T]
        sc = host_scalars(e, curve, 53 + spacing, sum(counts), dist, fmt)
        before = t.batch_commit(sc, counts, fmt=fmt)
        t.precompute(spacing)
        after = t.batch_commit(sc, counts, fmt=fmt)
        off = 0
        for i, c in enumerate(counts):
            a = after[i].x + after[i].y + after[i].z
            assert a == before[i].x + before[i].y + before[i].z, (i, c)
            if c:
                assert a == plain(e, curve, p, sc[off * 32:], fmt, c), (i, c)
            else:
                assert a == bytes(len(a))
            off += c
    finally:
        t.close()


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_shift_batch_matches_oracle(eng, oracles, curve):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    e = eng[curve]
    T = 512
    p, _ = gen_inputs(e, curve, 61, T, "uniform", zl.SCALAR_MONT)
    t = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        t.precompute(4)
        counts = [1, 37, 300, T]
        sc = host_scalars(e, curve, 62, sum(counts), "witness", zl.SCALAR_MONT)
        res = t.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)
        pts = to_host(p)
        off = 0
        for i, c in enumerate(counts):
            want = oracle_msm(orc, curve, pts, sc[off * 32:(off + c) * 32].tobytes(), c, zl.SCALAR_MONT)
            assert jac_to_affine_bytes(C, res[i].x + res[i].y + res[i].z) == want, (i, c)
            off += c
    finally:
        t.close()


def test_shift_spacing_change_and_drop(eng):
    e = eng["bn254"]
    T = 2048
    p, _ = gen_inputs(e, "bn254", 71, T, "uniform", zl.SCALAR_MONT)
    t = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        counts = [T, 999, 3]
        sc = host_scalars(e, "bn254", 72, sum(counts), "uniform", zl.SCALAR_MONT)
        base = [r.x + r.y + r.z for r in t.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)]
        for s in (8, 0, 3, 12):
            t.precompute(s)
            assert t.shift_bits == s
            got = [r.x + r.y + r.z for r in t.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)]
            assert got == base, s
        for bad in (1, 25, -1):
            with pytest.raises(MSMError):
                t.precompute(bad)
        assert t.shift_bits == 12
    finally:
        t.close()


def test_server_over_shift_tables(eng):
    """Served requests over shift tables equal the plain MSMs."""
    tabs, pts = {}, {}
    for curve, T in (("bn254", 1 << 13), ("bls12_381", 1 << 12)):
        p, _ = gen_inputs(eng[curve], curve, 81, T, "uniform", zl.SCALAR_MONT)
        tabs[curve] = CommitmentTable(eng[curve], p.data_ptr(), on_device=True, n=T)
        tabs[curve].precompute(4)
        pts[curve] = p
    srv = CommitmentServer(tabs["bn254"], tabs["bls12_381"], workers=2)
    try:
        reqs = []
        for j, (curve, n) in enumerate([("bn254", 1000), ("bls12_381", 300), ("bn254", 1 << 13), ("bn254", 5),
                                        ("bls12_381", 1 << 12), ("bn254", 64)]):
            sc = host_scalars(eng[curve], curve, 90 + j, n, "witness" if j % 2 else "uniform", zl.SCALAR_MONT)
            cid = zl.BN254 if curve == "bn254" else zl.BLS12_381
            reqs.append((curve, n, sc, srv.submit(cid, sc, zl.SCALAR_MONT)))
        for curve, n, sc, rid in reqs:
            res, _ = srv.wait(rid)
            assert res.x + res.y + res.z == plain(eng[curve], curve, pts[curve], sc, zl.SCALAR_MONT, n), (curve, n)
    finally:
        srv.close()
        for t in tabs.values():
            t.close()


@pytest.mark.parametrize("curve", ["bn254", "bls12_381"])
def test_shift_edge_cases(eng, curve):
    """Duplicate bases (the doubling path), cancellation, identity bases,
    zero and unreduced scalars and a hot bucket, over shift tables."""
    C = R.CURVES[curve]
    G = (C.gx, C.gy)
    P = R.scalar_mul(C, G, 987654321)
    Q = R.aff_neg(C, P)
    cases = [
        ([P, P, P], [3, 3, 3]),
        ([P, Q], [9, 9]),
        ([P, Q, P], [9, 9, 2]),
        ([None, P, None], [5, 7, 11]),
        ([P, G], [0, 0]),
        ([P, G], [1, 1]),
        ([P, G, P], [C.r - 1, C.r, C.r + 5]),
        ([P, G], [(1 << 256) - 1, (1 << 255)]),
        ([G] * 40, [1] * 40),
        ([P, P], [1 << 200, 1 << 200]),          # equal shifted copies in one bucket
    ]
    for pts, sc in cases:
        t = CommitmentTable(eng[curve], R.pack_points(C, pts))
        try:
            t.precompute(4)
            # two MSMs: the whole case, then its first point alone (one scalar each)
            r = t.batch_commit(R.pack_scalars_int(sc + sc[:1]), [len(pts), 1], fmt=zl.SCALAR_INT)
            assert jac_to_affine_bytes(C, r[0].x + r[0].y + r[0].z) == C.enc_affine(R.naive_msm(C, pts, sc)), \
                (pts, sc)
            assert jac_to_affine_bytes(C, r[1].x + r[1].y + r[1].z) == \
                C.enc_affine(R.naive_msm(C, pts[:1], sc[:1]))
        finally:
            t.close()
