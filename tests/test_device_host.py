"""Host-side helpers of the device set-up (no GPU): edge lists from adjacency lists and
networkx graphs in the node order of nx.to_numpy_array, and the time-grid test that chooses
between stepping one propagator and a batch of walks."""
import numpy as np

from fastctqw_b200.Operator import is_uniform_grid
from fastctqw_b200.device import edges_from_adjacency_list, edges_from_networkx


def _dense(n, edges):
    A = np.zeros((n, n))
    for u, v in edges:
        A[u, v] = A[v, u] = 1.0
    return A


def test_adjacency_list_edges_give_the_adjacency_matrix():
    rng = np.random.default_rng(0)
    A = np.triu(rng.random((30, 30)) < 0.2, 1)
    A = (A | A.T).astype(float)
    A[3, 3] = 1.0
    adj = [list(np.nonzero(A[u])[0]) for u in range(30)]
    e = edges_from_adjacency_list(adj)
    assert e.dtype == np.int64 and e.shape[1] == 2
    assert np.array_equal(_dense(30, e), A)
    assert edges_from_adjacency_list([[], []]).shape == (0, 2)


def test_networkx_edges_follow_to_numpy_array_order():
    import networkx as nx
    G = nx.Graph()
    G.add_nodes_from(["c", "a", "b", "d"])
    G.add_edges_from([("a", "b"), ("c", "d"), ("b", "c"), ("d", "d")])
    n, e = edges_from_networkx(G)
    assert n == 4
    assert np.array_equal(_dense(n, e), nx.to_numpy_array(G))


def test_uniform_grid_detection():
    assert is_uniform_grid(0.4 * np.arange(1, 21))
    assert is_uniform_grid([2.5])
    assert not is_uniform_grid([0.0, 1.0, 2.0])
    assert not is_uniform_grid([0.5, 1.0, 1.6])
    assert not is_uniform_grid([1.0, 2.0, 3.0 + 1e-9])
    assert not is_uniform_grid([])
