"""Multi-GPU layout of the benchmark: replicas only.  Each rank owns its own
ensemble (disjoint noise seeds, no data exchange) and the throughput is the
total points of all ranks over the max time over ranks.  Exercised here with
two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    ns, phis, c0s, ps = bench.ensemble(count=6, seed_base=rank * 6, rng_seed=rank)
    t = torch.tensor([1.0 + rank], dtype=torch.float64)          # this rank's "elapsed ms"
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    pts = torch.tensor([float(sum(n * n for n in ns))], dtype=torch.float64)
    dist.all_reduce(pts, op=dist.ReduceOp.SUM)
    q.put((rank, float(t.item()), float(pts.item()), [float(c.sum()) for c in c0s], ns))
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, t0, pts0, sums0, ns0), (r1, t1, pts1, sums1, ns1) = out
    assert t0 == t1 == 2.0                                     # max over ranks
    assert pts0 == pts1 == float(sum(n * n for n in ns0) + sum(n * n for n in ns1))
    assert sums0 != sums1                                      # disjoint seeds: different inputs


def test_ensemble_is_seeded_and_bounded():
    ns, phis, c0s, ps = bench.ensemble(count=8)
    ns2, phis2, c0s2, ps2 = bench.ensemble(count=8)
    assert ns == ns2 and all(np.array_equal(a, b) for a, b in zip(c0s, c0s2))
    assert set(ns) <= set(bench.SIZES)
    for p in ps:
        assert 2.5 <= p.P <= 10.0 and 0.25 <= p.chi <= 0.75 and 1.0 <= p.kappa <= 4.0
