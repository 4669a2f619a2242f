"""Continuous-time quantum walk, mirroring FastCTQW/Ctqw.py:6-97.

``runWalk(t)`` sets the final state to expm(-i H t) psi0 (Ctqw.py:90-94).  Here the product
U psi0 runs on the device right after the exponential, and only the N-vector psi crosses
back to the host (the reference copied the whole N x N U to the host for a numpy GEMV).

``from_networkx_graph`` accepts ``device`` and ``dtype`` keywords (a superset of the
reference signature, which could not take the ``device`` its README passes, README.md:64).
"""
from __future__ import annotations

import numpy as np

from .Operator import Operator, _check_device
from .State import State


class Ctqw:
    def __init__(self, data, initState: State, gamma: float = 1, laplacian: bool = False,
                 dtype=np.complex64, device: str = "cuda", ctqwId: str = "Undef") -> None:
        _check_device(device)
        self._device = device
        self.ctqwId = ctqwId
        self._initStator = initState
        if isinstance(data, Operator):
            self._n = data._n
            self._Operator = data
        elif isinstance(data, np.ndarray):
            self._n = data.shape[0]
            self._Operator = Operator.from_numpy_array(data, gamma, laplacian, device)
        elif isinstance(data, (int, np.integer)):
            self._n = int(data)
            self._Operator = Operator.from_num_nodes(self._n, dtype, device)
        else:
            raise TypeError(f"data must be an ndarray or an int, not {type(data).__name__}")
        self._finalStator = State.getSingleNodeState(self._n, 0) if self._n > 0 else None

    @classmethod
    def from_numpy_array(cls, A: np.ndarray, initState: State, gamma: float = 1,
                         laplacian: bool = False, ctqwId: str = "Undef",
                         device: str = "cuda") -> "Ctqw":
        return cls(A, initState, gamma, laplacian, device=device, ctqwId=ctqwId)

    @classmethod
    def from_networkx_graph(cls, graph, initState: State, gamma: float = 1,
                            laplacian: bool = False, ctqwId: str = "Undef", dtype=np.float32,
                            device: str = "cuda") -> "Ctqw":
        import networkx as nx
        if graph.is_directed():
            raise TypeError("graph is a directed graph, but Ctqw recive a undirected graph")
        return cls(nx.to_numpy_array(graph, dtype=dtype), initState, gamma, laplacian,
                   device=device, ctqwId=ctqwId)

    @classmethod
    def from_adjacency_list(cls, adj_list, initState: State, time: float = 1, gamma: float = 1,
                            laplacian: bool = False, ctqwId: str = "Undef", dtype=np.float32,
                            device: str = "cuda") -> "Ctqw":
        """Walk on the undirected graph ``adj_list[u]`` = neighbours of u, with H built on the
        device from the edges (FastCTQW/Ctqw.py:60-71 declares this constructor, with the same
        parameters, but leaves it empty; ``time`` is accepted for that signature and unused)."""
        return cls(Operator.from_adjacency_list(adj_list, gamma, laplacian, device, dtype), initState,
                   device=device, ctqwId=ctqwId)

    @classmethod
    def from_num_nodes(cls, n: int, initState: State | None = None, dtype=np.complex64,
                       device: str = "cuda") -> "Ctqw":
        return cls(n, initState, dtype=dtype, device=device)

    def reset_numpy_array(self, A: np.ndarray, initState: State, gamma: float = 1,
                          laplacian: bool = False):
        self._n = A.shape[0]
        self._Operator.reset_numpy_array(A, gamma, laplacian)
        self._initStator = initState
        self._finalStator = State.getSingleNodeState(self._n, 0)

    def reset_networkx_graph(self, nx_graph, initState: State, gamma: float = 1,
                             laplacian: bool = False):
        import networkx as nx
        self.reset_numpy_array(nx.to_numpy_array(nx_graph), initState, gamma, laplacian)

    def runWalk(self, time: float = 0):
        psi = self._Operator.propagate(time, self._initStator.getState())
        self._finalStator.setState(psi.astype(np.complex64, copy=False))

    def runWalks(self, times, markNodes=None, method: str = "auto") -> np.ndarray:
        """Probabilities at the marked nodes (all nodes when None) for every time: shape
        (len(times), len(markNodes)), the ``target_state`` that ``Plot.timeCurve`` plots
        (FastCTQW/Plot.py:35-49).  The final state becomes the state at the last time.  See
        ``Operator.time_curve`` for ``method``."""
        probs = self._Operator.time_curve(times, self._initStator.getState(), markNodes, method)
        last = getattr(self._Operator, "_last_state", None)
        if last is not None:
            self._finalStator.setState(last.cpu().numpy().astype(np.complex64, copy=False))
        return probs

    def getFinalState(self) -> State:
        return self._finalStator

    def getOperator(self):
        return self._Operator

    def free(self):
        self._Operator.free()
