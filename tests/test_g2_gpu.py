"""BN254 G2 MSM (GPU) against the Python restatement of the reference's G2
path (oracle/pyref.py G2Curve) and group identities (r*G2 = O, linearity,
k*G2 known answers), and against the reference itself through its compiled
C pairing: the reference has no C G2 MSM, but with bases k_i*G2 an MSM equals
t*G2 for a known t, and e(G1, MSM) = e(t*G1, G2) under the reference's
bn254_pairing pins each result (test_g2_msm_pinned_by_reference_pairing)."""
import ctypes
import random

import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import check, to_host
from zkmetal_b200 import BN254G2MSM, CommitmentTable
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu
G2 = R.BN254_G2


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return BN254G2MSM()


def aff(res):
    """Library result (X, Y, Z = 1 or identity (1, 1, 0)) -> affine point."""
    if not any(res.z):
        return None
    assert res.z == G2.enc_fp2((1, 0)), "library returns Z = 1 for finite points"
    return (G2.dec_fp2(res.x), G2.dec_fp2(res.y))


def scalars_bytes(sc):
    return R.pack_scalars_int(sc)


def test_g2_known_answers(eng):
    G = (G2.gx, G2.gy)
    for k in (1, 2, 5, 469, G2.r - 1, G2.r, G2.r + 3, (1 << 256) - 1):
        got = aff(eng.msm(G2.enc_affine(G), scalars_bytes([k])))
        assert got == G2.scalar_mul(G, k), k


def test_g2_small_vs_restatement(eng):
    rng = random.Random(21)
    for n, dist in ((1, "u"), (7, "u"), (33, "u"), (40, "w")):
        pts = G2.make_bases(21 + n, n)
        if dist == "u":
            sc = [rng.randrange(1 << 256) for _ in range(n)]
        else:
            sc = [0 if u < 40 else 1 if u < 60 else rng.getrandbits(32) if u < 85 else rng.randrange(G2.r)
                  for u in (rng.randrange(100) for _ in range(n))]
        got = aff(eng.msm(G2.pack_points(pts), scalars_bytes(sc)))
        assert got == G2.naive_msm(pts, sc), (n, dist)


def test_g2_edge_cases(eng):
    G = (G2.gx, G2.gy)
    P = G2.scalar_mul(G, 987654321)
    Q = G2.neg(P)
    cases = [([P, P, P], [3, 3, 3]), ([P, Q], [9, 9]), ([None, P, None], [5, 7, 11]), ([P, G], [0, 0]),
             ([G] * 40, [1] * 40), ([P, G, P], [G2.r - 1, G2.r, G2.r + 5])]
    for pts, sc in cases:
        assert aff(eng.msm(G2.pack_points(pts), scalars_bytes(sc))) == G2.naive_msm(pts, sc), (pts, sc)


def test_g2_montgomery_scalars(eng):
    rng = random.Random(5)
    pts = G2.make_bases(5, 16)
    sc = [rng.randrange(G2.r) for _ in range(16)]
    got = aff(eng.msmFr(G2.pack_points(pts), R.pack_scalars_mont(R.BN254, sc)))
    assert got == G2.naive_msm(pts, sc)


def test_g2_generator_and_split_linearity(eng):
    """Device-generated G2 bases equal the restatement's k_i * G2; an MSM of
    2^14 points equals the sum of the MSMs of its halves."""
    L = zl.lib()
    n = 1 << 14
    pts = torch.empty(n * 128, dtype=torch.uint8, device="cuda")
    sc = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(L.zkmsm_gen_bases(eng.handle, zl.BN254_G2, 31, 0, n, pts.data_ptr()))
    check(L.zkmsm_gen_scalars(eng.handle, zl.BN254_G2, 32, 0, n, 0, 1, sc.data_ptr()))
    host = to_host(pts)
    for i in (0, 1, 777, n - 1):
        assert G2.dec_affine(host[i * 128:(i + 1) * 128]) == G2.scalar_mul((G2.gx, G2.gy), R.base_scalar(G2, 31, i))

    def run(p, s, m):
        out = ctypes.create_string_buffer(192)
        torch.cuda.synchronize()
        check(L.zkmsm_msm_device(eng.handle, zl.BN254_G2, p.data_ptr(), s.data_ptr(), 1, m, out, None))
        raw = out.raw
        return aff(type("P", (), {"x": raw[:64], "y": raw[64:128], "z": raw[128:]}))

    full = run(pts, sc, n)
    h = n // 2
    a = run(pts[:h * 128], sc[:h * 32], h)
    b = run(pts[h * 128:], sc[h * 32:], h)
    assert full == G2.add(a, b)
    assert G2.on_curve(full)


def test_g2_table_batches_with_shifts(eng):
    """Batched MSMs over a resident G2 table, without and with window shifts."""
    T = 2048
    pts = G2.make_bases(41, 64) * (T // 64)
    rng = random.Random(41)
    counts = [1, 64, 333, T]
    sc = [rng.randrange(G2.r) for _ in range(sum(counts))]
    t = CommitmentTable(eng, G2.pack_points(pts))
    try:
        before = t.batch_commit(scalars_bytes(sc), counts)
        t.precompute(4)
        after = t.batch_commit(scalars_bytes(sc), counts)
        off = 0
        for i, c in enumerate(counts):
            assert before[i].x + before[i].y + before[i].z == after[i].x + after[i].y + after[i].z
            if c <= 64:
                assert aff(after[i]) == G2.naive_msm(pts[:c], sc[off:off + c]), c
            off += c
    finally:
        t.close()


@pytest.mark.parametrize("n", [4096, 1 << 16])
def test_g2_msm_pinned_by_reference_pairing(eng, oracles, n):
    """The device G2 MSM against the reference itself through its pairing:
    bases are k_i*G2 from the library's generator (k_i known from the
    restatement of the generator), so MSM(Q, s) = t*G2 with t = sum s_i k_i,
    and e(G1, MSM) must equal e(t*G1, G2) with the reference's bn254_pairing
    and bn254_point_scalar_mul (bn254_pairing.c:1320, bn254_msm.c:1333)."""
    ref, _ = oracles
    if ref is None or not ref.has_pairing:
        pytest.skip("reference C library not built")
    C = R.BN254
    L = zl.lib()
    seed = 977
    p = torch.empty(n * 128, dtype=torch.uint8, device="cuda")
    s = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(L.zkmsm_gen_bases(eng.handle, zl.BN254_G2, seed, 0, n, p.data_ptr()))
    check(L.zkmsm_gen_scalars(eng.handle, zl.BN254_G2, seed + 1, 0, n, 0, zl.SCALAR_INT, s.data_ptr()))
    sh = to_host(s)
    got = aff(eng.msm(to_host(p), sh))
    sc = [int.from_bytes(sh[32 * i:32 * i + 32], "little") for i in range(n)]
    t = sum(a * R.base_scalar(G2, seed, i) for i, a in enumerate(sc)) % G2.r
    G1b = C.enc_affine((C.gx, C.gy))
    lhs = ref.bn254_pairing(G1b, G2.enc_affine(got))
    rhs = ref.bn254_pairing(ref.point_scalar_mul("bn254", G1b, t), G2.enc_affine((G2.gx, G2.gy)))
    assert lhs == rhs
