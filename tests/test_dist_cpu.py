"""The N > 1 paths on the CPU with gloo, world size 2 (no GPU): bench.py's
rank plumbing (process group, barrier, max over ranks) and the batch split
across ranks with its all-gather of energies and gradients."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_runner(evals, gradients):
    # stands in for the device batch: energy = -n, gradient = parameter index + n / 100
    e = [-float(c.NumQubits()) for c, names, h, x in evals]
    g = [np.arange(len(names)) + c.NumQubits() / 100.0 for c, names, h, x in evals]
    return e, g


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    from goqu_b200 import batch, workloads
    try:
        w, r, _ = bench.dist_setup("gloo")
        bench.barrier(w)
        mx = bench.max_over_ranks(float(r + 1) * 1.5, w)
        evals = workloads.qaoa_batch(12, seed=3, n_values=(10, 12, 14))
        e, g = batch.run_sharded(evals, r, w, runner=_fake_runner)
        q.put((r, w, mx, e.tolist(), [x.tolist() for x in g]))
    finally:
        dist.destroy_process_group()


def test_two_rank_plumbing_and_sharded_batch():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from goqu_b200 import workloads
    evals = workloads.qaoa_batch(12, seed=3, n_values=(10, 12, 14))
    want_e, want_g = _fake_runner(evals, True)
    for r, w, mx, e, g in res:
        assert w == 2 and mx == 3.0
        assert np.allclose(e, want_e)
        assert all(np.allclose(a, b) for a, b in zip(g, want_g))


def test_split_by_work_balances_size_and_depth():
    from goqu_b200 import batch, workloads
    evals = workloads.qaoa_batch(200, seed=5)
    shares = batch.split_by_work(evals, 4)
    assert sorted(i for s in shares for i in s) == list(range(200))
    w = [batch.circuit_work(e) for e in evals]
    work = [sum(w[i] for i in s) for s in shares]
    assert max(work) - min(work) <= max(w)  # within one of the largest items
    # depth counts: circuits of equal size but four times the layers weigh about four times as much
    deep = [e for e in evals if e[0].NumQubits() == 20]
    p_of = [len(e[1]) // 2 for e in deep]
    w1 = [batch.circuit_work(e) for e, p in zip(deep, p_of) if p == 1]
    w4 = [batch.circuit_work(e) for e, p in zip(deep, p_of) if p == 4]
    if w1 and w4:
        assert 3.0 < min(w4) / max(w1) < 4.5
