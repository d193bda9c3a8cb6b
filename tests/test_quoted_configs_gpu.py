"""Parity at the sizes the benchmark configurations are quoted on (GPU).

Each device result is compared bit for bit, after normalising to affine, with
the reference's own C Pippenger compiled for the host (bn254_pippenger_msm,
bn254_msm.c:1145-1187; bls12_381_g1_pippenger_msm, bls12_381_ops.c:1141-1165)
on the same seeded inputs:

* BN254 G1, 2^24 points, uniform and witness-like Montgomery scalars (the
  headline configuration);
* BLS12-381 G1, 2^22 points, and each output of a batch of 8 MSMs with sizes
  log-uniform in [2^14, 2^22] over prefixes of the 2^22-point table;
* each output of the 24-MSM BN254 batch (sizes log-uniform in [2^12, 2^22],
  prefixes of a 2^22-point resident table), without and with the table's
  window shifts;
* a served stream of mixed BN254 / BLS12-381 requests.

The batch sizes are drawn exactly as the benchmark draws them.  When the
reference could not be compiled (no reference checkout and no prebuilt
library) the C restatement stands in.  Marked slow: the host Pippenger takes
seconds per case.
"""
import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import check, gen_inputs, jac_to_affine_bytes, msm_device, to_host
from zkmetal_b200 import BLS12381MSM, CommitmentServer, CommitmentTable, MetalMSM
from zkmetal_b200 import lib as zl

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    e = {"bn254": MetalMSM(), "bls12_381": BLS12381MSM()}
    yield e
    for x in e.values():
        x.close()


def ref_of(oracles):
    ref, cm = oracles
    return ref if ref is not None else cm


def gen_scalars(engine, curve, seed, n, dist, fmt):
    """Host bytes of the generator's scalars; the integer and Montgomery forms
    of one seed hold the same values."""
    s = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(zl.lib().zkmsm_gen_scalars(engine.handle, 0 if curve == "bn254" else 1, seed, 0, n,
                                     0 if dist == "uniform" else 1, fmt, s.data_ptr()))
    return to_host(s)


def int_scalars(engine, curve, seed, n, dist):
    return gen_scalars(engine, curve, seed, n, dist, zl.SCALAR_INT)


def ref_affine(orc, curve, points_b, scalars_int_b, n):
    return orc.msm(curve, points_b, scalars_int_b, n)


@pytest.mark.parametrize("dist", ["uniform", "witness"])
def test_bn254_2p24_vs_reference_c(eng, oracles, dist):
    orc = ref_of(oracles)
    C = R.BN254
    n = 1 << 24
    e = eng["bn254"]
    p, s = gen_inputs(e, "bn254", 0x5EED0001, n, dist, zl.SCALAR_MONT)
    got = jac_to_affine_bytes(C, msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n))
    ph, sh = to_host(p), to_host(s)
    del p, s
    torch.cuda.empty_cache()
    want = ref_affine(orc, "bn254", ph, orc.fr_from_mont("bn254", sh, n), n)
    assert got == want
    assert C.on_curve(C.dec_affine(got))


def test_bls12_381_2p22_plain_and_batch_of_8_vs_reference_c(eng, oracles):
    orc = ref_of(oracles)
    C = R.BLS12_381
    e = eng["bls12_381"]
    T = 1 << 22
    seed = 0x5EED0003
    rng = np.random.default_rng(seed)
    counts = [int(round(2 ** u)) for u in rng.uniform(14, 22, 8)]
    total = max(sum(counts), T)
    p = torch.empty(T * 96, dtype=torch.uint8, device="cuda")
    s = torch.empty(total * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(zl.lib().zkmsm_gen_bases(e.handle, 1, seed, 0, T, p.data_ptr()))
    check(zl.lib().zkmsm_gen_scalars(e.handle, 1, seed + 1, 0, total, 0, zl.SCALAR_MONT, s.data_ptr()))
    si = int_scalars(e, "bls12_381", seed + 1, total, "uniform")
    ph = to_host(p)
    # plain 2^22
    got = jac_to_affine_bytes(C, msm_device(e, "bls12_381", p, s, zl.SCALAR_MONT, T))
    assert got == ref_affine(orc, "bls12_381", ph, si[:T * 32], T)
    # batch of 8 over the resident table, then every output against the reference
    table = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        res = table.batch_commit(to_host(s)[:sum(counts) * 32], counts, fmt=zl.SCALAR_MONT)
        off = 0
        for i, (c, r) in enumerate(zip(counts, res)):
            want = ref_affine(orc, "bls12_381", ph[:c * 96], si[off * 32:(off + c) * 32], c)
            assert jac_to_affine_bytes(C, r.x + r.y + r.z) == want, (i, c)
            off += c
    finally:
        table.close()


def test_bn254_24_msm_batch_vs_reference_c(eng, oracles):
    """The 24 outputs of the batched configuration, with and without the
    resident table's window shifts (spacing 4 bits, the benchmark's)."""
    orc = ref_of(oracles)
    C = R.BN254
    e = eng["bn254"]
    T = 1 << 22
    seed = 0x5EED0002
    rng = np.random.default_rng(seed)
    counts = [int(round(2 ** u)) for u in rng.uniform(12, 22, 24)]
    total = sum(counts)
    p = torch.empty(T * 64, dtype=torch.uint8, device="cuda")
    s = torch.empty(total * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    check(zl.lib().zkmsm_gen_bases(e.handle, 0, seed, 0, T, p.data_ptr()))
    check(zl.lib().zkmsm_gen_scalars(e.handle, 0, seed + 1, 0, total, 0, zl.SCALAR_MONT, s.data_ptr()))
    si = int_scalars(e, "bn254", seed + 1, total, "uniform")
    ph, sh = to_host(p), np.frombuffer(to_host(s), dtype=np.uint8)
    want, off = [], 0
    for c in counts:
        want.append(ref_affine(orc, "bn254", ph[:c * 64], si[off * 32:(off + c) * 32], c))
        off += c
    table = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        for shifts in (0, 4):
            if shifts:
                table.precompute(shifts)
            for on_device in (False, True):
                res = table.batch_commit(s.data_ptr() if on_device else sh, counts, fmt=zl.SCALAR_MONT,
                                         on_device=on_device)
                got = [jac_to_affine_bytes(C, r.x + r.y + r.z) for r in res]
                bad = [i for i in range(len(counts)) if got[i] != want[i]]
                assert not bad, (shifts, on_device, bad)
    finally:
        table.close()


def test_served_stream_vs_reference_c(eng, oracles):
    """A mixed stream (BN254 and BLS12-381, uniform and witness-like scalars,
    sizes 2^8..2^20) through the continuous-batching server over window-shift
    tables, all submitted before the first wait so requests share batches;
    every result against the reference C Pippenger of its request."""
    orc = ref_of(oracles)
    T = 1 << 20
    seed = 0x5EED0004
    rng = np.random.default_rng(seed)
    tabs, hosts, pools, ints = {}, {}, {}, {}
    try:
        for ci, curve in enumerate(("bn254", "bls12_381")):
            fb = R.CURVES[curve].fp_bytes
            p = torch.empty(T * 2 * fb, dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            check(zl.lib().zkmsm_gen_bases(eng[curve].handle, ci, seed + ci, 0, T, p.data_ptr()))
            tabs[curve] = CommitmentTable(eng[curve], p.data_ptr(), on_device=True, n=T)
            tabs[curve].precompute(4)
            hosts[curve] = to_host(p)
            for dist in ("uniform", "witness"):
                pools[(curve, dist)] = np.frombuffer(
                    gen_scalars(eng[curve], curve, seed + 10 + ci, T, dist, zl.SCALAR_MONT), dtype=np.uint8).copy()
                ints[(curve, dist)] = int_scalars(eng[curve], curve, seed + 10 + ci, T, dist)
        srv = CommitmentServer(tabs["bn254"], tabs["bls12_381"], workers=3)
        reqs = []
        for _ in range(40):
            curve = "bn254" if rng.random() < 0.7 else "bls12_381"
            dist = "uniform" if rng.random() < 0.5 else "witness"
            n = int(round(2 ** rng.uniform(8, 20)))
            reqs.append((curve, dist, n))
        ids = [srv.submit(0 if c == "bn254" else 1, pools[(c, d)][:n * 32], zl.SCALAR_MONT) for c, d, n in reqs]
        out = [srv.wait(i)[0] for i in ids]
        srv.close()
        for (curve, dist, n), r in zip(reqs, out):
            C = R.CURVES[curve]
            want = ref_affine(orc, curve, hosts[curve][:n * 2 * C.fp_bytes], ints[(curve, dist)][:n * 32], n)
            assert jac_to_affine_bytes(C, r.x + r.y + r.z) == want, (curve, dist, n)
    finally:
        for t in tabs.values():
            t.close()
