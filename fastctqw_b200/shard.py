"""A batch of independent walks over the ranks of a process group (one process per GPU).

The walks do not interact, so the batch shards with no collective in the data path: every rank
computes the same greedy longest-processing-time partition of the walks by their cost, runs its
share through one ``WalkBatch`` on its own GPU, and rank 0 gathers the states at the end (the
one collective, ``gather_object``; NCCL over NVLink between GPUs, gloo on CPU).

Cost of a walk: the algorithm's flop count F(N, m, s) = 8 N^3 (pi_m + s) + (8/3) N^3 + 8 N^3,
with m = 13 and s estimated from the exact 1-norm of X (s = max(0, ceil(log2(||X||_1 /
theta_13)))), the same first-order estimate the Al-Mohy & Higham selection starts from.
"""
from __future__ import annotations

import math

import numpy as np

PADE_PRODUCTS = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}
THETA_13 = 4.25


def walk_cost(n: int, s: int, m: int = 13) -> float:
    """F(N, m, s) in flops (one generic complex GEMM = 8 N^3)."""
    n3 = float(n) ** 3
    return 8.0 * n3 * (PADE_PRODUCTS[m] + s) + (8.0 / 3.0) * n3 + 8.0 * n3


def estimate_s(X: np.ndarray) -> int:
    """Squarings from the exact 1-norm of X (host, one pass)."""
    norm1 = float(np.abs(X).sum(axis=0).max()) if X.size else 0.0
    if norm1 <= THETA_13:
        return 0
    return int(math.ceil(math.log2(norm1 / THETA_13)))


def partition_lpt(costs, world: int):
    """Greedy longest-processing-time: walks by decreasing cost, each to the least-loaded rank
    (ties to the lower index, so every rank computes the same partition).  Returns the walk
    indices of each rank (ascending) and the ranks' loads."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(p) for p in parts], loads


def _walkbatch_runner(Xs, psi0s):
    from .batch import WalkBatch
    with WalkBatch([X.shape[0] for X in Xs], Xs[0].dtype) as b:
        return b.run(Xs, psi0s)


def run_sharded(Xs, psi0s=None, group=None, runner=None, costs=None):
    """psi_w = expm(X_w) psi0_w for all walks, sharded over the ranks of ``group``.

    Every rank passes the same ``Xs`` (and ``psi0s``).  Returns the list of states on rank 0
    and None elsewhere; without an initialised process group it runs everything locally.
    ``runner(Xs_share, psi0s_share) -> states`` defaults to one ``WalkBatch`` on this rank's
    GPU; ``costs`` defaults to ``walk_cost(N, estimate_s(X))``."""
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if dist_on else 0
    world = dist.get_world_size(group) if dist_on else 1
    if costs is None:
        costs = [walk_cost(X.shape[0], estimate_s(X)) for X in Xs]
    parts, _ = partition_lpt(costs, world)
    mine = parts[rank]
    runner = runner or _walkbatch_runner
    local = runner([Xs[i] for i in mine], [psi0s[i] for i in mine] if psi0s is not None else None) if mine else []
    payload = [(i, np.asarray(p)) for i, p in zip(mine, local)]
    if not dist_on:
        gathered = [payload]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
        if rank != 0:
            return None
    out = [None] * len(Xs)
    for part in gathered:
        for i, psi in part:
            out[i] = psi
    return out
