"""The allocation-free BN254 entry point, checked against the engine entry point.

zkmsm_bn254_msm_noalloc exists for callers that cannot call cudaMalloc (a
framework that has reserved nearly all device memory for its own pool, or a
hot loop that forbids allocation after start-up).  Its scratch is one static
device array shared by all calls, so this test makes several calls in a row
on different inputs -- each must match the existing device entry point
(zkmsm_msm_device) bit for bit, showing the shared scratch is re-initialised
between calls -- queues calls back to back on one stream with no wait between
them (the documented way to reuse the scratch), checks one result directly
against the oracle, and checks that bad arguments and sizes above the limit
are refused with an error message.

Collected last on purpose (file name) so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process (it creates its own engine and inputs).
"""
import ctypes

import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import check, gen_inputs, jac_to_affine_bytes, msm_device, oracle_msm, to_host
from zkmetal_b200 import MetalMSM
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu

LIMIT = 8192


@pytest.fixture(scope="module")
def engine():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = MetalMSM()
    yield e
    e.close()


def noalloc(d_points, d_scalars, fmt, n):
    out = torch.zeros(96, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(zl.lib().zkmsm_bn254_msm_noalloc(d_points.data_ptr(), d_scalars.data_ptr(), fmt, n, out.data_ptr(), None))
    torch.cuda.synchronize()
    return out.cpu().numpy().tobytes()


def test_noalloc_matches_engine_on_consecutive_calls(engine):
    cases = [(LIMIT, "uniform", zl.SCALAR_MONT, 901), (3000, "witness", zl.SCALAR_INT, 902),
             (1, "uniform", zl.SCALAR_MONT, 903), (LIMIT, "uniform", zl.SCALAR_MONT, 901)]
    for n, dist, fmt, seed in cases:
        p, s = gen_inputs(engine, "bn254", seed, n, dist, fmt)
        want = msm_device(engine, "bn254", p, s, fmt, n)
        got = noalloc(p, s, fmt, n)
        assert got == want, (n, dist, fmt)


def test_noalloc_calls_queued_on_one_stream(engine):
    """Three calls on different inputs queued on one stream with no wait in
    between: the stream orders them, so each clears and reuses the scratch
    after the previous call is done with it."""
    cases = [(LIMIT, "uniform", zl.SCALAR_MONT, 911), (2500, "witness", zl.SCALAR_MONT, 912),
             (4097, "uniform", zl.SCALAR_INT, 913)]
    inputs = [gen_inputs(engine, "bn254", seed, n, dist, fmt) for n, dist, fmt, seed in cases]
    outs = [torch.zeros(96, dtype=torch.uint8, device="cuda") for _ in cases]
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for (n, _, fmt, _), (p, s), out in zip(cases, inputs, outs):
        check(zl.lib().zkmsm_bn254_msm_noalloc(p.data_ptr(), s.data_ptr(), fmt, n, out.data_ptr(),
                                               ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    for (n, dist, fmt, _), (p, s), out in zip(cases, inputs, outs):
        assert out.cpu().numpy().tobytes() == msm_device(engine, "bn254", p, s, fmt, n), (n, dist, fmt)


def test_noalloc_matches_oracle(engine, oracles):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    n = 3000
    p, s = gen_inputs(engine, "bn254", 921, n, "witness", zl.SCALAR_MONT)
    got = jac_to_affine_bytes(R.BN254, noalloc(p, s, zl.SCALAR_MONT, n))
    assert got == oracle_msm(orc, "bn254", to_host(p), to_host(s), n, zl.SCALAR_MONT)


def test_noalloc_rejects_sizes_above_limit(engine):
    p, s = gen_inputs(engine, "bn254", 904, 16, "uniform", zl.SCALAR_MONT)
    out = torch.zeros(96, dtype=torch.uint8, device="cuda")
    st = zl.lib().zkmsm_bn254_msm_noalloc(p.data_ptr(), s.data_ptr(), zl.SCALAR_MONT, LIMIT + 1, out.data_ptr(), None)
    assert st == zl.ERR_INVALID_INPUT
    assert "8192" in zl.last_error()
    assert zl.lib().zkmsm_bn254_msm_noalloc(None, s.data_ptr(), 0, 4, out.data_ptr(), None) == zl.ERR_INVALID_INPUT
    assert "null" in zl.last_error()
    assert zl.lib().zkmsm_bn254_msm_noalloc(p.data_ptr(), s.data_ptr(), 7, 4, out.data_ptr(), None) == \
        zl.ERR_INVALID_INPUT
    assert "scalar_fmt" in zl.last_error()
    assert zl.lib().zkmsm_bn254_msm_noalloc(p.data_ptr(), s.data_ptr(), 0, 0, out.data_ptr(), None) == \
        zl.ERR_INVALID_INPUT
    assert "n_points is 0" in zl.last_error()
