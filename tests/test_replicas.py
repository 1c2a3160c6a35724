"""The multi-GPU form (query-sharded replicas) on CPU gloo ranks: distinct
query batches per rank, max-over-ranks step timing, whole-job value, and the
oracle answering each rank's batch on its own (no exchange needed)."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from fknn import datagen, replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vecs, labels, ts = datagen.make_base(3000, 1.1, 1000, 1235)
        q, m = replicas.rank_queries(1, 16, rank)
        ids, _ = oracle.exact_knn(vecs, labels, ts, q, m, nthreads=1)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        slowest = replicas.max_over_ranks(ms)
        out.put((rank, q.sum(), ids[:, 0].tolist(), slowest, replicas.job_value(world, 16, slowest)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, f0, m0, v0), (r1, s1, f1, m1, v1) = res
    assert s0 != s1                      # each rank has its own batch
    assert m0 == m1 == 15.0              # both see the slowest rank's time
    assert v0 == v1 == 2 * 16 / 0.015    # whole-job queries/s
    q0, _ = replicas.rank_queries(1, 16, 0)
    w = datagen.WORKLOADS[1]
    q_ref, _ = datagen.make_queries(16, w.zipf_s, w.n_labels, w.window, w.balanced_types, 1235, 1236)
    np.testing.assert_array_equal(q0, q_ref)  # rank 0 answers the workload's own queries


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_value(1, 100, 20.0) == 5000.0
