"""CPU tests of the oracle itself: the Python and C restatements against the
golden vectors made with the reference's compiled C Pippenger, against each
other, and against the reference's own known-answer shapes
(Tests/zkMetalTests/MSMTests.swift:7-62, DASTests.swift:8-150)."""
import hashlib
import json
import os
import random

import pytest

from oracle import pyref as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "msm_golden.json")


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.parametrize("case", golden()["cases"], ids=lambda c: "%s-%d-%d-%s" % (c["curve"], c["seed"], c["n"], c["dist"]))
def test_golden_cases(case, oracles):
    ref, cm = oracles
    C = R.CURVES[case["curve"]]
    pts = R.make_bases(C, case["seed"], case["n"])
    sc = R.make_scalars(C, case["seed"], case["n"], case["dist"])
    pb, sb = R.pack_points(C, pts), R.pack_scalars_int(sc)
    assert hashlib.sha256(pb + sb).hexdigest() == case["input_sha256"], "input generator drifted"
    want = bytes.fromhex(case["result_affine"])
    assert cm.msm(C.name, pb, sb, case["n"]) == want
    if ref is not None:
        assert ref.msm(C.name, pb, sb, case["n"]) == want
    if case["n"] <= 64:
        assert C.enc_affine(R.naive_msm(C, pts, sc)) == want
        assert C.enc_affine(R.glv_signed_msm(C, pts, sc, 5)) == want


@pytest.mark.parametrize("kat", golden()["kat"], ids=lambda k: "%s-%s" % (k["curve"], k["name"]))
def test_golden_kats(kat, oracles):
    _, cm = oracles
    C = R.CURVES[kat["curve"]]
    pb = b"".join(bytes.fromhex(p) for p in kat["points"])
    sb = R.pack_scalars_int(kat["scalars"])
    assert cm.msm(C.name, pb, sb, len(kat["scalars"])) == bytes.fromhex(kat["result_affine"])


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_edge_cases_restatements_agree(curve, oracles):
    """Duplicate bases, P + (-P), identity bases, zero / one / r-1 / 2^256-1
    scalars: cases the reference tests do not cover."""
    ref, cm = oracles
    C = R.CURVES[curve]
    G = (C.gx, C.gy)
    P = R.scalar_mul(C, G, 123456789)
    negP = R.aff_neg(C, P)
    pts = [P, P, negP, G, P, G, negP, P]
    sc = [5, 5, 10, 0, 1, C.r - 1, C.r - 1, (1 << 256) - 1]
    want = R.naive_msm(C, pts, sc)
    pb, sb = R.pack_points(C, pts), R.pack_scalars_int(sc)
    assert C.dec_affine(cm.msm(curve, pb, sb, len(pts))) == want
    if ref is not None:
        assert C.dec_affine(ref.msm(curve, pb, sb, len(pts))) == want
    assert R.glv_signed_msm(C, pts, [s % C.r for s in sc], 4) == want
    # cancelling to the identity
    pts2, sc2 = [P, negP], [7, 7]
    assert R.naive_msm(C, pts2, sc2) is None
    assert cm.msm(curve, R.pack_points(C, pts2), R.pack_scalars_int(sc2), 2) == bytes(2 * C.fp_bytes)


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_glv_split_bound(curve):
    """k = k1 + k2*lambda (mod r) and |k_i| < 2^HALF_BITS over random and
    edge scalars (the bound fixes the signed window count)."""
    C = R.CURVES[curve]
    bits = R.glv_half_bits(C)
    rng = random.Random(7)
    ks = [0, 1, 2, C.r - 1, C.r - 2, C.lam, C.r - C.lam, C.r // 2, C.r // 2 + 1, (1 << 127), (1 << 128) - 1]
    g = C.glv
    for v in (g["a1"], g["a2"], g["b1"], g["b2"]):
        ks += [abs(v) % C.r, (C.r - abs(v)) % C.r, (abs(v) * C.lam) % C.r]
    ks += [rng.randrange(C.r) for _ in range(20000)]
    for k in ks:
        k1, k2 = R.glv_split(C, k)
        assert (k1 + k2 * C.lam - k) % C.r == 0
        assert abs(k1) < (1 << bits) and abs(k2) < (1 << bits)


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_glv_split_bound_1e7_in_c(curve, oracles):
    """The same bound over 4*10^7 seeded uniform scalars, by the oracle's C
    restatement of the split (exact 256/512-bit integer arithmetic),
    cross-checked against the Python split on the edge scalars and 2000
    random ones.  k1 + k2*lambda = k (mod r) holds for any c1, c2 because
    the lattice vectors satisfy a + b*lambda = 0 (mod r), checked once in
    the constant derivation."""
    _, cm = oracles
    C = R.CURVES[curve]
    bits = R.glv_half_bits(C)
    rng = random.Random(11)
    ks = [0, 1, 2, C.r - 1, C.r - 2, C.lam, C.r - C.lam, C.r // 2] + [rng.randrange(C.r) for _ in range(2000)]
    want = max(max(abs(a).bit_length(), abs(b).bit_length()) for a, b in (R.glv_split(C, k) for k in ks))
    assert cm.glv_max_bits(curve, C.glv, 0, 0, ks) == want
    assert cm.glv_max_bits(curve, C.glv, 0x61C, 4 * 10 ** 7) <= bits


def test_endomorphism_constants():
    for C in (R.BN254, R.BLS12_381, R.BLS12_377):
        assert pow(C.beta, 3, C.p) == 1 and C.beta != 1
        assert (C.lam * C.lam + C.lam + 1) % C.r == 0
        G = (C.gx, C.gy)
        Q = R.scalar_mul(C, G, 987654321)
        assert R.scalar_mul(C, Q, C.lam) == (C.beta * Q[0] % C.p, Q[1])


@pytest.mark.parametrize("c", [2, 3, 5, 8, 13, 16, 19, 22])
def test_signed_digits_roundtrip(c):
    rng = random.Random(c)
    for _ in range(2000):
        bits = rng.choice([1, 8, 32, 127, 128, 255])
        k = rng.getrandbits(bits)
        nw = (bits + 1 + c - 1) // c
        ds = R.signed_digits(k, c, nw)
        assert sum(d << (c * j) for j, d in enumerate(ds)) == k
        assert all(-(1 << (c - 1)) <= d <= (1 << (c - 1)) for d in ds)


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_montgomery_fr_conversion(curve, oracles):
    ref, cm = oracles
    C = R.CURVES[curve]
    sc = R.make_scalars(C, 3, 50, "uniform") + [0, 1, C.r - 1]
    mont = R.pack_scalars_mont(C, sc)
    assert cm.fr_from_mont(curve, mont, len(sc)) == R.pack_scalars_int(sc)
    if ref is not None:
        assert ref.fr_from_mont(curve, mont, len(sc)) == R.pack_scalars_int(sc)


def test_witness_distribution_shape():
    C = R.BN254
    sc = R.make_scalars(C, 99, 4000, "witness")
    zeros = sum(s == 0 for s in sc) / len(sc)
    ones = sum(s == 1 for s in sc) / len(sc)
    small = sum(1 < s < (1 << 32) for s in sc) / len(sc)
    assert 0.36 < zeros < 0.44 and 0.17 < ones < 0.23 and 0.21 < small < 0.29


def test_c_restatement_matches_reference_medium(oracles):
    """Both C oracles on a 2^12 input (window widths 11-13 paths)."""
    ref, cm = oracles
    if ref is None:
        pytest.skip("reference C oracle not built (no reference checkout)")
    C = R.BN254
    n = 4096
    rng = random.Random(5)
    G = (C.gx, C.gy)
    base = R.scalar_mul(C, G, 77)
    # cheap distinct bases: P_i = (i+1)*base by repeated addition (as MSMTests.swift:13-16)
    pts, acc = [], base
    for _ in range(n):
        pts.append(acc)
        acc = R.aff_add(C, acc, base)
    sc = [rng.randrange(1 << 256) for _ in range(n)]
    pb, sb = R.pack_points(C, pts), R.pack_scalars_int(sc)
    assert cm.msm("bn254", pb, sb, n) == ref.msm("bn254", pb, sb, n)


def test_g2_restatement_group_laws():
    """BN254 G2 restatement: generator on the twist, order r, additivity,
    encoding round trip."""
    G2 = R.BN254_G2
    G = (G2.gx, G2.gy)
    assert G2.on_curve(G)
    assert G2.scalar_mul(G, G2.r) is None
    P = G2.scalar_mul(G, 1234567)
    assert G2.add(P, G2.neg(P)) is None
    assert G2.add(G2.scalar_mul(G, 5), G2.scalar_mul(G, 7)) == G2.scalar_mul(G, 12)
    assert G2.dec_affine(G2.enc_affine(P)) == P
    assert G2.enc_affine(None) == bytes(128)


@pytest.mark.parametrize("curve", ["bn254", "bls12_381", "bls12_377"])
def test_host_generator_matches_restatement(curve, oracles):
    """The oracle's C generator (used for the CPU-only reference inputs) gives
    the same bytes as the Python restatement of the seeded generator, which
    the library's device generator matches (test_generator_matches_restatement):
    scalars in both forms and distributions, and bases k_i*G from the comb."""
    _, cm = oracles
    C = R.CURVES[curve]
    for dist in ("uniform", "witness"):
        sc = [R.scalar_uniform(C, 77, i) if dist == "uniform" else R.scalar_witness(C, 77, i) for i in range(5, 45)]
        assert cm.gen_scalars(curve, 77, 40, dist, 0, index0=5).tobytes() == R.pack_scalars_int(sc)
        assert cm.gen_scalars(curve, 77, 40, dist, 1, index0=5).tobytes() == R.pack_scalars_mont(C, sc)
    got = cm.gen_bases(curve, C.enc_affine((C.gx, C.gy)), 77, 24, index0=3).tobytes()
    assert got == R.pack_points(C, [R.scalar_mul(C, (C.gx, C.gy), R.base_scalar(C, 77, i)) for i in range(3, 27)])


def test_g2_restatement_pinned_by_reference_pairing(oracles):
    """The BN254 G2 restatement (the checker of the G2 MSM) against the
    reference's own optimal ate pairing (bn254_pairing, bn254_pairing.c:1320):
    with bases Q_i = k_i*G2, MSM(Q, s) = t*G2 for t = sum s_i k_i, so
    e(G1, MSM) must equal e(t*G1, G2), t*G1 by the reference's
    bn254_point_scalar_mul.  The reference has no C G2 MSM; bilinearity of its
    pairing pins the G2 results to it."""
    ref, _ = oracles
    if ref is None or not ref.has_pairing:
        pytest.skip("reference C library not built")
    C, G2 = R.BN254, R.BN254_G2
    G1b = C.enc_affine((C.gx, C.gy))
    Q = (G2.gx, G2.gy)
    rng = random.Random(23)
    for n in (1, 3, 17):
        ks = [R.base_scalar(G2, 55, i) for i in range(n)]
        pts = [G2.scalar_mul(Q, k) for k in ks]
        sc = [rng.randrange(G2.r) for _ in range(n)]
        t = sum(a * b for a, b in zip(sc, ks)) % G2.r
        msm = G2.naive_msm(pts, sc)
        lhs = ref.bn254_pairing(G1b, G2.enc_affine(msm))
        rhs = ref.bn254_pairing(ref.point_scalar_mul("bn254", G1b, t), G2.enc_affine(Q))
        assert lhs == rhs, n
    assert ref.bn254_pairing(G1b, G2.enc_affine(G2.scalar_mul(Q, 2))) != ref.bn254_pairing(G1b, G2.enc_affine(Q))
