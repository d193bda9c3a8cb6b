"""Base-field arithmetic of the CUDA kernels, checked word for word.

The product and square the MSM kernels use (even/odd-split CIOS Montgomery
product) and the straight CIOS product are run through zkmsm_field_op on
random operands below 2p and on edge values, and compared with a*b/R mod p
computed with Python integers.
The reference's field code is the Montgomery CIOS in
NeonFieldOps/bn254_msm.c:38-267 and Shaders/fields/bn254_fp.metal:134-233.
"""
import random

import numpy as np
import pytest
import torch

from oracle import pyref as R
from zkmetal_b200 import lib as zl

CASES = [("bn254", R.BN254, 8, zl.BN254), ("bls12_381", R.BLS12_381, 12, zl.BLS12_381),
         ("bls12_377", R.BLS12_377, 12, zl.BLS12_377)]


def _limbs(vals, n):
    out = np.zeros((len(vals), n), dtype=np.uint32)
    for i, v in enumerate(vals):
        for l in range(n):
            out[i, l] = (v >> (32 * l)) & 0xFFFFFFFF
    return out


def _ints(arr):
    return [sum(int(w) << (32 * l) for l, w in enumerate(row)) for row in arr]


@pytest.mark.gpu
@pytest.mark.parametrize("name,C,n_limbs,curve", CASES)
def test_field_mul_sqr_match_integers(name, C, n_limbs, curve):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = C.p
    rinv = pow(1 << (32 * n_limbs), -1, p)
    rng = random.Random(0xF1E1D + curve)
    edge = [0, 1, 2, p - 1, p - 2, p, p + 1, 2 * p - 1, (1 << 32) - 1, (1 << 64) - 1, p >> 1, (p + 1) // 2,
            (1 << (p.bit_length() - 1)), (1 << (32 * (n_limbs // 2))) - 1, (1 << (32 * (n_limbs // 2)))]
    edge = [e for e in edge if e < 2 * p]
    xs = [a for a in edge for _ in edge] + [rng.randrange(2 * p if i % 2 else p) for i in range(6000)]
    ys = [b for _ in edge for b in edge] + [rng.randrange(2 * p if i % 3 else p) for i in range(6000)]
    n = len(xs)
    da = torch.from_numpy(_limbs(xs, n_limbs)).cuda()
    db = torch.from_numpy(_limbs(ys, n_limbs)).cuda()
    out = torch.empty_like(da)
    L = zl.lib()
    for op in (0, 1, 2):
        assert L.zkmsm_field_op(curve, op, da.data_ptr(), db.data_ptr(), out.data_ptr(), n) == 0
        got = _ints(out.cpu().numpy())
        for i in range(n):
            want = (xs[i] * (xs[i] if op == 1 else ys[i]) * rinv) % p
            assert got[i] == want, (name, op, i, hex(xs[i]), hex(ys[i]))


def test_field_op_rejects_bad_arguments():
    """Argument checks happen before any device work (runs without a GPU)."""
    L = zl.lib()
    assert L.zkmsm_field_op(0, 7, 1, 1, 1, 1) == zl.ERR_INVALID_INPUT
    assert L.zkmsm_field_op(5, 0, 1, 1, 1, 1) == zl.ERR_INVALID_INPUT
    assert L.zkmsm_field_op(0, 0, None, 1, 1, 1) == zl.ERR_INVALID_INPUT
