"""Multi-rank plumbing of the sharded MSM on CPU (gloo, world size 2).

Each rank computes the partial MSM of its point range (here with the C
oracle, since these ranks have no GPU), the partials are all-gathered in rank
order and added; the sum must equal the MSM over all points.  This covers the
shard boundaries, the gather and the combination that bench.py --gpus N runs
over NCCL with the CUDA library doing the partial MSMs and the addition.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import pyref as R
from zkmetal_b200.shard import gather_partials, shard_range, sharded_msm


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, curve_name, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.lib import COracle
        C = R.CURVES[curve_name]
        cm = COracle()
        pts = R.make_bases(C, 77, n)
        sc = R.make_scalars(C, 77, n, "witness")
        f = C.fp_bytes

        def partial(start, stop):
            aff = cm.msm(curve_name, R.pack_points(C, pts[start:stop]), R.pack_scalars_int(sc[start:stop]),
                         stop - start) if stop > start else bytes(2 * f)
            return torch.frombuffer(bytearray(aff), dtype=torch.uint8)

        def add(gathered, w):
            acc = bytes(2 * f)
            raw = gathered.numpy().tobytes()
            for g in range(w):
                acc = cm.affine_add(curve_name, acc, raw[g * 2 * f:(g + 1) * 2 * f])
            return acc

        got = sharded_msm(n, world, rank, partial, add)
        # rank order of the gather
        tag = torch.tensor([rank], dtype=torch.int64)
        order = gather_partials(tag, world).tolist()
        q.put((rank, got, order, C.enc_affine(R.naive_msm(C, pts, sc)) if rank == 0 else None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("curve_name,n", [("bn254", 37), ("bls12_381", 11)])
def test_sharded_msm_gloo_world2(curve_name, n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, curve_name, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    want = res[0][3]
    assert res[0][1] == res[1][1] == want
    assert res[0][2] == res[1][2] == [0, 1]
