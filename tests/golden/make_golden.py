#!/usr/bin/env python3
"""Generate tests/golden/msm_golden.json from the reference's own C Pippenger.

Each case is defined by (curve, seed, n, distribution); its inputs are
regenerated deterministically by oracle/pyref.py (bases k_i*G, scalars uniform
in Fr or witness-like), and the expected affine result is computed here by the
reference's compiled C Pippenger (oracle/_ref/libzkref.so, built from the
reference sources by oracle/build_ref.py) and, for the small cases, also by a
naive double-and-add sum.  A SHA-256 of the packed inputs is stored so a
change to the generator is caught instead of silently changing the inputs.

Also stored: the known-answer shapes of the reference tests
(Tests/zkMetalTests/MSMTests.swift:7-62, DASTests.swift:8-150): 5*G,
MSM([G, 42G], [7, 11]) = 469*G on BLS12-381, 16-point zero-padded version,
scalar 0 -> identity, scalar 1 -> point; BLS12-377 cases from the reference's
bls12_377_g1_pippenger_msm (NeonFieldOps/bls12_377_ops.c:1476).

Run (needs the reference checkout to build the C oracle):
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build as obuild  # noqa: E402
from oracle import lib as olib  # noqa: E402
from oracle import pyref as R  # noqa: E402

CASES = [
    # curve, seed, n, dist, also_naive
    ("bn254", 11, 1, "uniform", True),
    ("bn254", 12, 7, "uniform", True),
    ("bn254", 13, 64, "uniform", True),
    ("bn254", 14, 64, "witness", True),
    ("bn254", 15, 300, "uniform", False),
    ("bn254", 16, 1000, "witness", False),
    ("bls12_381", 21, 1, "uniform", True),
    ("bls12_381", 22, 40, "uniform", True),
    ("bls12_381", 23, 40, "witness", True),
    ("bls12_381", 24, 200, "uniform", False),
    ("bls12_377", 31, 1, "uniform", True),
    ("bls12_377", 32, 40, "uniform", True),
    ("bls12_377", 33, 40, "witness", True),
    ("bls12_377", 34, 200, "uniform", False),
]


def case_inputs(C, seed, n, dist):
    pts = R.make_bases(C, seed, n)
    sc = R.make_scalars(C, seed, n, dist)
    return pts, sc


def digest(pb, sb):
    return hashlib.sha256(pb + sb).hexdigest()


def main():
    obuild.build_all()
    ref = olib.RefOracle()
    out = {"cases": [], "kat": []}
    for curve, seed, n, dist, naive in CASES:
        C = R.CURVES[curve]
        pts, sc = case_inputs(C, seed, n, dist)
        pb, sb = R.pack_points(C, pts), R.pack_scalars_int(sc)
        res = ref.msm(curve, pb, sb, n)
        if naive:
            want = R.naive_msm(C, pts, sc)
            assert C.dec_affine(res) == want, (curve, seed)
        out["cases"].append(dict(curve=curve, seed=seed, n=n, dist=dist, input_sha256=digest(pb, sb),
                                 result_affine=res.hex(), checked_naive=naive))
        print(curve, seed, n, dist, res.hex()[:16])
    # known answers
    for C in (R.BN254, R.BLS12_381, R.BLS12_377):
        G = (C.gx, C.gy)
        five = R.scalar_mul(C, G, 5)
        out["kat"].append(dict(curve=C.name, name="5G", points=[C.enc_affine(G).hex()], scalars=[5],
                               result_affine=C.enc_affine(five).hex()))
    C = R.BLS12_381
    G = (C.gx, C.gy)
    srs = [R.scalar_mul(C, G, pow(42, i, C.r)) for i in range(16)]
    want = C.enc_affine(R.scalar_mul(C, G, 469))
    got = ref.msm(C.name, R.pack_points(C, srs[:2]), R.pack_scalars_int([7, 11]), 2)
    assert got == want
    out["kat"].append(dict(curve=C.name, name="SRS42[:2]*[7,11]=469G", points=[C.enc_affine(P).hex() for P in srs[:2]],
                           scalars=[7, 11], result_affine=want.hex()))
    sc16 = [7, 11] + [0] * 14
    got16 = ref.msm(C.name, R.pack_points(C, srs), R.pack_scalars_int(sc16), 16)
    assert got16 == want
    out["kat"].append(dict(curve=C.name, name="SRS42[:16]*[7,11,0..]=469G", points=[C.enc_affine(P).hex() for P in srs],
                           scalars=sc16, result_affine=want.hex()))
    for C in (R.BN254, R.BLS12_381, R.BLS12_377):
        G = (C.gx, C.gy)
        out["kat"].append(dict(curve=C.name, name="0*G=identity", points=[C.enc_affine(G).hex()], scalars=[0],
                               result_affine=C.enc_affine(None).hex()))
        P3 = R.scalar_mul(C, G, 3)
        out["kat"].append(dict(curve=C.name, name="1*3G=3G", points=[C.enc_affine(P3).hex()], scalars=[1],
                               result_affine=C.enc_affine(P3).hex()))
    with open(os.path.join(HERE, "msm_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "msm_golden.json"))


if __name__ == "__main__":
    main()
