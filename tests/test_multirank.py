"""Multi-rank scenario sharding on CPU: two gloo ranks each solve their shard of a batch with
the FP64 oracle (standing in for one GPU each) and gather the results, which must equal a
single-process solve of the whole batch."""

import os
import socket

import numpy as np
import pytest


def test_shard_covers_everything_once():
    from gap_b200.sharding import shard

    for n, w in ((10, 3), (1024, 8), (5, 8)):
        got = np.concatenate([shard(n, w, r) for r in range(w)])
        assert np.array_equal(np.sort(got), np.arange(n))
    costs = np.r_[np.full(4, 10.0), np.ones(12)]
    loads = [costs[shard(16, 2, r, costs)].sum() for r in range(2)]
    assert abs(loads[0] - loads[1]) <= 1.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import torch.distributed as dist

    from gap_b200 import synth
    from gap_b200.sharding import gather, shard
    from oracle import restate

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    net = synth.feeder_grid(1, n=60)
    S = 7
    s_spec = synth.load_scenarios(net, S, sigma=0.1, seed=3, base_power=1e6)
    idx = shard(S, world, rank)
    v = np.zeros((len(idx), net.n_bus), np.complex128)
    it = np.zeros(len(idx), np.int64)
    for j, s in enumerate(idx):
        o = restate.nr_solve(net, tol=1e-10, max_iter=30, base_power=1e6, s_spec=s_spec[s])
        v[j] = o["v"]
        it[j] = o["iterations"]
    full = gather(idx, {"v": v, "iterations": it}, S)
    if rank == 0:
        np.savez(out_path, **full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_serial_result(tmp_path):
    import multiprocessing as mp

    from gap_b200 import synth
    from oracle import restate

    port = _free_port()
    out = str(tmp_path / "full.npz")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    full = np.load(out)
    net = synth.feeder_grid(1, n=60)
    s_spec = synth.load_scenarios(net, 7, sigma=0.1, seed=3, base_power=1e6)
    for s in range(7):
        o = restate.nr_solve(net, tol=1e-10, max_iter=30, base_power=1e6, s_spec=s_spec[s])
        np.testing.assert_allclose(full["v"][s], o["v"], atol=1e-14)
        assert full["iterations"][s] == o["iterations"]
