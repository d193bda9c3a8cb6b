"""Batched commitments, autotuner and the commitment server (GPU).

Every batched or served result must equal, bit for bit, the plain single
MSM of the same scalars over the same table prefix.  The server's failure
paths are exercised on the host only (admission refusal, cancellation,
injected batch failures): nothing here faults or stalls the GPU.
"""
import ctypes
import json
import random

import numpy as np
import pytest
import torch

from oracle import pyref as R
from tests.gpu_helpers import check, gen_inputs, jac_to_affine_bytes, msm_device, oracle_msm, to_host
from zkmetal_b200 import BLS12381MSM, CommitmentServer, CommitmentTable, MetalMSM, MSMError
from zkmetal_b200 import lib as zl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return {"bn254": MetalMSM(), "bls12_381": BLS12381MSM()}


@pytest.fixture(scope="module")
def tables(eng):
    out = {}
    for curve, T in (("bn254", 1 << 15), ("bls12_381", 1 << 13)):
        p, _ = gen_inputs(eng[curve], curve, 301, T, "uniform", zl.SCALAR_MONT)
        out[curve] = (CommitmentTable(eng[curve], p.data_ptr(), on_device=True, n=T), p)
    yield out
    for t, _ in out.values():
        t.close()


def scalars_host(eng, curve, seed, n, dist):
    _, s = gen_inputs(eng, curve, seed, n, dist, zl.SCALAR_MONT)
    return np.frombuffer(to_host(s), dtype=np.uint8).copy()


def plain(eng, curve, table_points, scal_np, n):
    s = torch.from_numpy(scal_np[: n * 32].copy()).cuda()
    return msm_device(eng, curve, table_points, s, zl.SCALAR_MONT, n)


def test_batch_graph_replay_and_launch_count(eng, tables):
    e = eng["bn254"]
    table, pts = tables["bn254"]
    counts = [4096, 100, 1 << 15, 1, 777]
    sc = scalars_host(e, "bn254", 310, sum(counts), "witness")
    L = zl.lib()
    r1 = table.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)  # launches issued directly
    l0 = L.zkmsm_engine_launch_count(e.handle)
    r2 = table.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)  # captured into a graph
    l1 = L.zkmsm_engine_launch_count(e.handle)
    r3 = table.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)  # replayed graph
    l2 = L.zkmsm_engine_launch_count(e.handle)
    assert l1 > l0 and l2 - l1 == l1 - l0
    off = 0
    for i, c in enumerate(counts):
        a = r1[i].x + r1[i].y + r1[i].z
        assert a == r2[i].x + r2[i].y + r2[i].z == r3[i].x + r3[i].y + r3[i].z
        assert a == plain(e, "bn254", pts, sc[off * 32:], c)
        off += c


def test_autotune_keeps_results_and_persists(eng, oracles, tmp_path):
    ref, cm = oracles
    orc = ref if ref is not None else cm
    e = MetalMSM()
    L = zl.lib()
    buf = ctypes.create_string_buffer(1 << 16)
    check(L.zkmsm_autotune(e.handle, zl.BN254, 10, 13, buf, len(buf)))
    rep = json.loads(buf.value.decode())
    assert set(rep) == {"10", "11", "12", "13"}
    for v in rep.values():
        assert str(v["best"]) in v["ms"]
    n = 3000
    p, s = gen_inputs(e, "bn254", 320, n, "uniform", zl.SCALAR_MONT)
    got = jac_to_affine_bytes(R.BN254, msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n))
    assert got == oracle_msm(orc, "bn254", to_host(p), to_host(s), n, zl.SCALAR_MONT)
    path = str(tmp_path / "tuning.txt")
    check(L.zkmsm_tuning_save(e.handle, path.encode()))
    e2 = MetalMSM()
    check(L.zkmsm_tuning_load(e2.handle, path.encode()))
    assert msm_device(e2, "bn254", p, s, zl.SCALAR_MONT, n) == msm_device(e, "bn254", p, s, zl.SCALAR_MONT, n)
    with open(path) as f:
        assert f.readline().startswith("zkmsm-tuning")
    e.close()
    e2.close()


def test_server_same_result_alone_and_in_the_mix(eng, tables):
    srv = CommitmentServer(tables["bn254"][0], tables["bls12_381"][0], workers=2)
    try:
        rng = random.Random(5)
        pool = {c: scalars_host(eng[c], c, 330 + i, tables[c][0].n, "uniform" if i else "witness")
                for i, c in enumerate(("bn254", "bls12_381"))}
        cid = {"bn254": zl.BN254, "bls12_381": zl.BLS12_381}
        probe = ("bn254", 5000)
        rid = srv.submit(cid["bn254"], pool["bn254"][: probe[1] * 32], zl.SCALAR_MONT)
        alone, lat = srv.wait(rid)
        assert lat > 0
        reqs = []
        for k in range(40):
            curve = "bn254" if rng.random() < 0.7 else "bls12_381"
            n = int(2 ** rng.uniform(4, np.log2(tables[curve][0].n)))
            reqs.append((curve, n))
            if k == 17:
                reqs.append(probe)
        ids = [srv.submit(cid[c], pool[c][: n * 32], zl.SCALAR_MONT) for c, n in reqs]
        res = [srv.wait(i)[0] for i in ids]
        for (c, n), r in zip(reqs, res):
            want = plain(eng[c], c, tables[c][1], pool[c], n)
            assert r.x + r.y + r.z == want, (c, n)
        k = reqs.index(probe)
        assert res[k].x + res[k].y + res[k].z == alone.x + alone.y + alone.z
        st = srv.stats()
        assert st["completed"] >= 42 and st["failed"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0
    finally:
        srv.close()


def test_server_admission_cancel_and_injected_failure(eng, tables):
    t = tables["bn254"][0]
    pool = scalars_host(eng["bn254"], "bn254", 340, t.n, "uniform")
    small = CommitmentServer(t, None, hbm_budget_bytes=32 << 20, workers=1)
    try:
        with pytest.raises(MSMError):
            small.submit(zl.BN254, pool[: t.n * 32], zl.SCALAR_MONT)  # needs more than the budget
    finally:
        small.close()
    srv = CommitmentServer(t, None, workers=1, max_batch_points=1 << 12)
    try:
        srv.inject_failures(1)
        first = srv.submit(zl.BN254, pool[: 2000 * 32], zl.SCALAR_MONT)
        with pytest.raises(MSMError):
            srv.wait(first)
        ids = [srv.submit(zl.BN254, pool[: 3000 * 32], zl.SCALAR_MONT) for _ in range(12)]
        cancelled = ids[-1]
        st = srv.cancel(cancelled)
        assert st in (zl.SUCCESS, zl.ERR_BUSY)  # BUSY if it had already started
        for i in ids[:-1]:
            r, _ = srv.wait(i)
            assert r.x + r.y + r.z == plain(eng["bn254"], "bn254", tables["bn254"][1], pool, 3000)
        if st == zl.SUCCESS:
            with pytest.raises(MSMError):
                srv.wait(cancelled)
        else:
            srv.wait(cancelled)
        assert srv.stats()["failed"] == 1
    finally:
        srv.close()


def test_server_large_batch_matches_plain(eng):
    """A batch above the small-batch limit (2^20 points) runs on the worker's
    normal-priority stream; its results match plain MSMs of the same scalars."""
    e = eng["bn254"]
    T = (1 << 20) + 4096
    p, _ = gen_inputs(e, "bn254", 350, T, "uniform", zl.SCALAR_MONT)
    table = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    srv = CommitmentServer(table, None, workers=1)
    try:
        sc = scalars_host(e, "bn254", 351, T, "witness")
        ids = [srv.submit(zl.BN254, sc[: n * 32], zl.SCALAR_MONT) for n in (T, 1000, T - 5)]
        res = [srv.wait(i)[0] for i in ids]
        for (n, r) in zip((T, 1000, T - 5), res):
            assert r.x + r.y + r.z == plain(e, "bn254", p, sc, n), n
    finally:
        srv.close()
        table.close()


@pytest.mark.parametrize("shift", [0, 4])
def test_grouped_batch_from_host_scalars(eng, shift):
    """A batch of host scalars large enough to run as groups (copy of group g
    + 1 overlapping group g) equals the plain MSMs, with and without window
    shifts, zero counts included."""
    e = eng["bn254"]
    T = 1 << 22
    p, _ = gen_inputs(e, "bn254", 141, T, "uniform", zl.SCALAR_MONT)
    counts = [T, 1 << 19, 3, 0, T, 777, 0]   # over 2^23 points: two groups
    sc = scalars_host(e, "bn254", 142, sum(counts), "witness")
    table = CommitmentTable(e, p.data_ptr(), on_device=True, n=T)
    try:
        if shift:
            table.precompute(shift)
        res = table.batch_commit(sc, counts, fmt=zl.SCALAR_MONT)
    finally:
        table.close()
    off = 0
    for i, c in enumerate(counts):
        got = res[i].x + res[i].y + res[i].z
        if c == 0:
            assert got == bytes(96)
        else:
            assert got == plain(e, "bn254", p, sc[off * 32:], c), (i, c)
        off += c


def test_replica_pool_routes_and_matches_plain(eng):
    """Two replicas (servers with their own tables; both on device 0 here, one
    per GPU in production) behind one pool: requests are spread over both
    and every result equals the plain MSM of its request."""
    from zkmetal_b200 import CommitmentServerPool
    T = 1 << 14
    reps, tabs, pts = [], [], {}
    try:
        for k in range(2):
            for curve, cid in (("bn254", 0), ("bls12_381", 1)):
                p, _ = gen_inputs(eng[curve], curve, 340 + cid, T, "uniform", zl.SCALAR_MONT)
                pts[curve] = p
                tabs.append(CommitmentTable(eng[curve], p.data_ptr(), on_device=True, n=T))
            reps.append(CommitmentServer(tabs[-2], tabs[-1], workers=2))
        pool = CommitmentServerPool(reps)
        rng = random.Random(5)
        reqs = []
        for i in range(40):
            curve = "bn254" if rng.random() < 0.7 else "bls12_381"
            n = rng.randint(1, T)
            reqs.append((curve, n, scalars_host(eng[curve], curve, 350 + i, n, "uniform" if i % 2 else "witness")))
        # all submitted before the first wait, so the replicas' queues fill
        ids = [pool.submit(0 if c == "bn254" else 1, sc, zl.SCALAR_MONT) for c, _, sc in reqs]
        for (curve, n, sc), rid in zip(reqs, ids):
            r, _ = pool.wait(rid)
            assert r.x + r.y + r.z == plain(eng[curve], curve, pts[curve], sc, n)
        st = pool.stats()
        assert [x["routed"] for x in st["replicas"]] and all(x["routed"] > 0 for x in st["replicas"])
        assert sum(x["completed"] for x in st["replicas"]) == 40
        pool.close()
    finally:
        for s in reps:
            s.close()
        for t in tabs:
            t.close()
