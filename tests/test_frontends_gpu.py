"""The batch front-ends of the reference's MultiMSM.swift (GPU), each result
against the oracle: multiMSM with integer and Fr scalar sets (:21-72),
multiMSMPipelined (:250), innerProductMSM with uneven and empty partitions
(:90-128), innerProductMSMHalves (:134-150) and batchMSMAsync over tasks of
different sizes and scalar forms (:155-246), plus their invalid-input cases
(MSMError("invalidInput") where the reference throws MSMError.invalidInput).
"""
import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import gen_inputs, jac_to_affine_bytes, oracle_msm, to_host
from zkmetal_b200 import (BLS12381MSM, MetalMSM, MSMError, MSMTask, batchMSMAsync, innerProductMSM,
                          innerProductMSMHalves, multiMSM, multiMSMPipelined)
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = {"bn254": MetalMSM(), "bls12_381": BLS12381MSM()}
    yield e
    for x in e.values():
        x.close()


def orc_of(oracles):
    ref, cm = oracles
    return ref if ref is not None else cm


def host_inputs(e, curve, seed, n, dist, fmt):
    p, s = gen_inputs(e, curve, seed, n, dist, fmt)
    return to_host(p), to_host(s)


def aff(curve, r):
    return jac_to_affine_bytes(R.CURVES[curve], r.x + r.y + r.z)


@pytest.mark.parametrize("curve", ["bn254", "bls12_381"])
def test_multi_msm_int_and_fr_sets(eng, oracles, curve):
    orc = orc_of(oracles)
    e = eng[curve]
    C = R.CURVES[curve]
    n = 3000
    ph, _ = host_inputs(e, curve, 601, n, "uniform", zl.SCALAR_INT)
    sets_int = [host_inputs(e, curve, 602 + k, n, "uniform" if k % 2 else "witness", zl.SCALAR_INT)[1]
                for k in range(3)]
    sets_fr = [host_inputs(e, curve, 602 + k, n, "uniform" if k % 2 else "witness", zl.SCALAR_MONT)[1]
               for k in range(3)]
    want = [oracle_msm(orc, curve, ph, s, n, zl.SCALAR_INT) for s in sets_int]
    assert [aff(curve, r) for r in multiMSM(e, ph, sets_int)] == want
    assert [aff(curve, r) for r in multiMSM(e, ph, frScalarSets=sets_fr)] == want
    assert [aff(curve, r) for r in multiMSMPipelined(e, ph, sets_int)] == want
    assert multiMSM(e, ph, []) == []
    with pytest.raises(MSMError) as ei:
        multiMSM(e, ph, [sets_int[0][:32 * (n - 1)]])
    assert ei.value.case == "invalidInput"
    assert C.fp_bytes == zl.FP_BYTES[e.curve]


def test_inner_product_msm_partitions(eng, oracles):
    orc = orc_of(oracles)
    e = eng["bn254"]
    n = 5000
    for fmt in (zl.SCALAR_INT, zl.SCALAR_MONT):
        ph, sh = host_inputs(e, "bn254", 611, n, "uniform", fmt)
        parts = [0, 1, 1, 2100, 2100, 4096, n]
        res = innerProductMSM(e, ph, sh, parts, fr=fmt == zl.SCALAR_MONT)
        assert len(res) == len(parts) - 1
        for (a, b), r in zip(zip(parts, parts[1:]), res):
            if a == b:
                # the reference's pointIdentity(): (1, 1, 0) with 1 in Montgomery form
                assert (r.x, r.y, r.z) == (zl.mont_one(zl.BN254), zl.mont_one(zl.BN254), bytes(32))
            else:
                assert aff("bn254", r) == oracle_msm(orc, "bn254", ph[a * 64:b * 64], sh[a * 32:b * 32], b - a, fmt)
        l, r = innerProductMSMHalves(e, ph, sh, fr=fmt == zl.SCALAR_MONT)
        h = n // 2
        assert aff("bn254", l) == oracle_msm(orc, "bn254", ph[:h * 64], sh[:h * 32], h, fmt)
        assert aff("bn254", r) == oracle_msm(orc, "bn254", ph[h * 64:], sh[h * 32:], n - h, fmt)
    for bad in ([0, n - 1], [1, n], [0], [0, 3000, 2000, n]):
        with pytest.raises(MSMError) as ei:
            innerProductMSM(e, ph, sh, bad)
        assert ei.value.case == "invalidInput"
    with pytest.raises(MSMError):
        innerProductMSMHalves(e, ph[:64], sh[:32])


@pytest.mark.parametrize("curve", ["bn254", "bls12_381"])
def test_batch_msm_async_mixed_tasks(eng, oracles, curve):
    orc = orc_of(oracles)
    e = eng[curve]
    sizes = [1, 2049, 17, 70000, 300]
    tasks, want = [], []
    for i, n in enumerate(sizes):
        fmt = zl.SCALAR_MONT if i % 2 else zl.SCALAR_INT
        ph, sh = host_inputs(e, curve, 620 + i, n, "witness" if i == 3 else "uniform", fmt)
        tasks.append(MSMTask(ph, frScalars=sh) if fmt == zl.SCALAR_MONT else MSMTask(ph, scalars=sh))
        want.append(oracle_msm(orc, curve, ph, sh, n, fmt))
    got = [aff(curve, r) for r in batchMSMAsync(e, tasks)]
    assert got == want
    assert batchMSMAsync(e, []) == []
    with pytest.raises(MSMError) as ei:
        batchMSMAsync(e, [MSMTask(tasks[1].points, scalars=np.zeros(32, dtype=np.uint8))])
    assert ei.value.case == "invalidInput"
