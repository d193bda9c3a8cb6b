"""Commitment front-end over a resident SRS (GPU): KZGEngine.commit /
batchCommit must equal the plain MSM of the same Fr coefficients over the
SRS prefix (and the oracle on a small case), batched or one by one."""
import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import gen_inputs, jac_to_affine_bytes, msm_device, oracle_msm, to_host
from zkmetal_b200 import BLS12381MSM, KZGEngine, MetalMSM, MSMError
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return {"bn254": MetalMSM(), "bls12_381": BLS12381MSM()}


@pytest.mark.parametrize("curve,shift", [("bn254", 4), ("bn254", 0), ("bls12_381", 4)])
def test_kzg_commit_matches_plain_msm(eng, oracles, curve, shift):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    C = R.CURVES[curve]
    e = eng[curve]
    T = 1 << 12
    p, _ = gen_inputs(e, curve, 121, T, "uniform", zl.SCALAR_MONT)
    srs = np.frombuffer(to_host(p), dtype=np.uint8).copy()
    kzg = KZGEngine(srs, engine=e, shift_bits=shift)
    try:
        assert kzg.srs_size == T
        lens = [1, 100, T, 333, 2]
        _, s = gen_inputs(e, curve, 122, sum(lens), "witness", zl.SCALAR_MONT)
        coeffs = np.frombuffer(to_host(s), dtype=np.uint8)
        polys, off = [], 0
        for n in lens:
            polys.append(coeffs[off * 32:(off + n) * 32].copy())
            off += n
        batch = kzg.batchCommit(polys)
        for poly, n, b in zip(polys, lens, batch):
            one = kzg.commit(poly)
            assert one.x + one.y + one.z == b.x + b.y + b.z
            plain = msm_device(e, curve, p, torch.from_numpy(poly).cuda(), zl.SCALAR_MONT, n)
            assert b.x + b.y + b.z == plain, n
        small = polys[1]
        assert jac_to_affine_bytes(C, batch[1].x + batch[1].y + batch[1].z) == \
            oracle_msm(orc, curve, to_host(p), small.tobytes(), 100, zl.SCALAR_MONT)
        with pytest.raises(MSMError):
            kzg.commit(np.zeros((T + 1) * 32, dtype=np.uint8))
        with pytest.raises(MSMError):
            kzg.commit(np.zeros(0, dtype=np.uint8))
        assert kzg.batchCommit([]) == []
    finally:
        kzg.close()
