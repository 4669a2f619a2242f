"""Seeded synthetic graph families for the walk workloads.

The reference takes graphs from networkx (``Ctqw.from_networkx_graph``,
FastCTQW/Ctqw.py:45-57) and its tests draw complete, G(n, 0.05) and random 4-regular
graphs (tests/test_fastexpm_accuracy.py:83-160).  These generators produce the same
families reproducibly from a seed, as dense float adjacency matrices:

* ``random_regular``: networkx ``random_regular_graph(d, n, seed)``.
* ``erdos_renyi``: upper-triangle Bernoulli(p) from ``numpy.random.default_rng(seed)``
  (networkx's G(10^4, 0.5) builder takes over a minute; this takes about a second).
* ``weighted_complete``: symmetric weights uniform in [0, 1), zero diagonal.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def random_regular(n: int, d: int, seed: int, dtype=np.float32) -> np.ndarray:
    import networkx as nx
    g = nx.random_regular_graph(d, n, seed=seed)
    return nx.to_numpy_array(g, dtype=dtype, nodelist=range(n))


def erdos_renyi(n: int, p: float, seed: int, dtype=np.float32) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n), dtype=dtype)
    iu = np.triu_indices(n, 1)
    a[iu] = (rng.random(iu[0].size) < p).astype(dtype)
    return a + a.T


def weighted_complete(n: int, seed: int, dtype=np.float32) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w = np.zeros((n, n), dtype=np.float64)
    iu = np.triu_indices(n, 1)
    w[iu] = rng.random(iu[0].size)
    return (w + w.T).astype(dtype)


def complete(n: int, dtype=np.float32) -> np.ndarray:
    return (np.ones((n, n)) - np.eye(n)).astype(dtype)


def laplacian(a: np.ndarray) -> np.ndarray:
    """D - A with D = diag(row sums), in A's dtype."""
    return (np.diag(a.sum(axis=1)) - a).astype(a.dtype)


def uniform_state(n: int) -> np.ndarray:
    return np.full(n, 1.0 / math.sqrt(n), dtype=np.complex64)


def basis_state(n: int, k: int = 0) -> np.ndarray:
    s = np.zeros(n, dtype=np.complex64)
    s[k] = 1.0
    return s


def random_state(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return (v / np.linalg.norm(v)).astype(np.complex64)


@dataclass
class WalkSpec:
    """One walk of an uneven batch: graph family, size, degree / edge probability, time."""
    kind: str
    n: int
    t: float
    d: int = 0
    p: float = 0.0
    seed: int = 0

    def adjacency(self, dtype=np.float32) -> np.ndarray:
        if self.kind == "regular":
            return random_regular(self.n, self.d, self.seed, dtype)
        return erdos_renyi(self.n, self.p, self.seed, dtype)


def uneven_batch(count: int = 512, seed: int = 3, nmin: int = 64, nmax: int = 2048,
                 tmin: float = 0.5, tmax: float = 50.0) -> list[WalkSpec]:
    """The uneven batch family: N ~ U{nmin..nmax}; alternating random d-regular
    (d ~ U{3..16}; when N*d is odd, d+1 is used) and G(N, p) with p ~ U[0.05, 0.5];
    t log-uniform in [tmin, tmax]."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        t = float(math.exp(rng.uniform(math.log(tmin), math.log(tmax))))
        if k % 2 == 0:
            d = int(rng.integers(3, 17))
            if (n * d) % 2:
                d += 1
            specs.append(WalkSpec("regular", n, t, d=d, seed=seed * 100003 + k))
        else:
            p = float(rng.uniform(0.05, 0.5))
            specs.append(WalkSpec("er", n, t, p=p, seed=seed * 100003 + k))
    return specs
