"""Sharding a batch of walks over ranks (CPU: gloo, world size 2; the oracle stands in for the
per-rank GPU batch).  Checks: the longest-processing-time partition covers every walk once,
is the same on every rank and is balanced; the gathered states equal a single-process run
bit for bit, also when a rank gets no walk."""
import os
import socket
import tempfile

import numpy as np
import pytest

from fastctqw_b200 import shard


def test_partition_covers_every_walk_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.random(53) ** 3 * 1e12)
    for world in (1, 2, 3, 8):
        parts, loads = shard.partition_lpt(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(53))
        assert parts == shard.partition_lpt(costs, world)[0]            # deterministic
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-3     # greedy list bound
        for p, ld in zip(parts, loads):
            assert abs(sum(costs[i] for i in p) - ld) <= 1e-6 * max(1.0, ld)
    parts, loads = shard.partition_lpt([5.0], 3)
    assert parts == [[0], [], []]


def test_cost_model_and_squaring_estimate():
    assert shard.walk_cost(10, 0, 13) == pytest.approx(8e3 * 6 + 8e3 / 3 + 8e3)
    assert shard.walk_cost(10, 4) > shard.walk_cost(10, 3) > shard.walk_cost(9, 3)
    X = np.zeros((4, 4), np.complex64)
    assert shard.estimate_s(X) == 0
    X[0, 1] = X[1, 0] = 1j * 100.0
    assert shard.estimate_s(X) == int(np.ceil(np.log2(100.0 / 4.25)))


def _walks(count, seed):
    rng = np.random.default_rng(seed)
    Xs, P = [], []
    for k in range(count):
        n = int(rng.integers(3, 40))
        A = np.triu(rng.random((n, n)) < 0.3, 1)
        A = (A | A.T).astype(np.float64)
        Xs.append(np.asarray(1j * A * rng.uniform(0.2, 5.0), np.complex128))
        p = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        P.append(p / np.linalg.norm(p))
    return Xs, P


def _oracle_runner(Xs, psi0s):
    from oracle import expm_oracle as eo
    return [eo.expm(X) @ p for X, p in zip(Xs, psi0s)]


def _rank_main(rank, world, port, count, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        Xs, P = _walks(count, 7)
        res = shard.run_sharded(Xs, P, runner=_oracle_runner)
        if rank == 0:
            np.savez(os.path.join(out_dir, "states.npz"), *res)
        else:
            assert res is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("count", [13, 1])
def test_gloo_two_ranks_match_one_process(count):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), count, d), nprocs=2, join=True,
                           start_method="spawn")
        got = np.load(os.path.join(d, "states.npz"))
        got = [got[f"arr_{i}"] for i in range(count)]
    Xs, P = _walks(count, 7)
    ref = _oracle_runner(Xs, P)
    assert len(got) == count
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


def test_without_a_process_group_everything_runs_locally():
    Xs, P = _walks(5, 3)
    got = shard.run_sharded(Xs, P, runner=_oracle_runner)
    for g, r in zip(got, _oracle_runner(Xs, P)):
        assert np.array_equal(g, r)
