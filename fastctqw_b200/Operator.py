"""Hamiltonian and propagator of a walk, mirroring FastCTQW/Operator.py:6-166.

``Operator(A, gamma, laplacian)`` checks that ``A`` is a symmetric adjacency matrix
(``ValueError`` otherwise, :80-90), picks complex64 for float32/complex64 data and
complex128 for float64/complex128 data (``TypeError`` otherwise, :27-32), builds
H = -gamma A or -gamma (D - A) (:49-53), checks that H is Hermitian (:92-103), and
``buildExpmOperator(t)`` computes U = expm(-i H t) (:70-78).

Differences from the reference, all deliberate:
* the exponential always runs on the B200 engine; ``device`` other than "cuda" raises
  ``ValueError`` (there is no CPU fallback),
* the engine dtype follows the data dtype (the reference built a complex64 engine from its
  ``dtype`` argument even for float64 data, :40, :58-66),
* ``propagate(t, psi0)`` returns U psi0 without copying U to the host; ``getOperator()``
  fetches U lazily afterwards,
* ``from_num_nodes`` / ``reset_networkx_graph`` pass their arguments to the right
  parameters (the reference mixed them up, :118-120, :144-146),
* ``from_adjacency_list`` (a stub in the reference, :115-117) keeps the graph as an edge list
  on the device and builds X = -i H t there for every time (``fastctqw_b200.device``); no
  N x N host matrix is made,
* ``time_curve(times, psi0, nodes)`` gives the probabilities of a walk at many times: one
  propagator stepped along a uniform grid, or one grouped batch of walks otherwise.
"""
from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

from .fastexpm import ExpMatComplex64, ExpMatComplex128


def is_uniform_grid(times) -> bool:
    """True when times are t_k = (k + 1) t_0 (k = 0, 1, ...) with t_0 > 0, to 1e-12 relative:
    the grid on which one propagator U(t_0) can be stepped."""
    times = np.asarray(times, dtype=np.float64).reshape(-1)
    if times.size == 0 or not times[0] > 0:
        return False
    return bool(np.allclose(times, times[0] * np.arange(1, times.size + 1), rtol=1e-12, atol=0.0))


def _check_device(device: str) -> None:
    if device != "cuda":
        raise ValueError("fastctqw_b200 computes on the B200 only: use device='cuda'")


class Operator:
    def __init__(self, data, gamma: float = 1, laplacian: bool = False, device: str = "cuda",
                 dtype=np.complex64) -> None:
        _check_device(device)
        self._device = device
        self._expmMat = None
        self._walked = False
        self._edges = None
        if isinstance(data, np.ndarray):
            if not self._is_adjacency_matrix(data):
                raise ValueError("A is not a adj matrix")
            self._n = data.shape[0]
            self._gamma = gamma
            self._laplacian = laplacian
            self._dtype = self._dtype_for(data)
            self._hamiltonian = self._buildHamiltonian(data, gamma)
            if not self._is_hermitian(self._hamiltonian):
                raise ValueError("_hamiltonian is not a hamiltonian matrix")
            self._expMator = self._initExpMator(self._n, self._dtype)
        elif isinstance(data, (int, np.integer)):
            self._n = int(data)
            self._dtype = np.dtype(dtype).type
            self._expMator = self._initExpMator(self._n, self._dtype)
        else:
            raise TypeError(f"data must be an ndarray or an int, not {type(data).__name__}")

    @staticmethod
    def _dtype_for(A: np.ndarray):
        if A.dtype in (np.float32, np.complex64):
            return np.complex64
        if A.dtype in (np.float64, np.complex128):
            return np.complex128
        raise TypeError(f"A.dtype is error : {A.dtype}")

    def free(self):
        self._expMator.free()

    def _buildHamiltonian(self, A: np.ndarray, gamma: float) -> NDArray:
        if self._laplacian:
            return -gamma * np.asarray(np.diag(A.sum(axis=1)) - A, dtype=self._dtype)
        return -gamma * np.asarray(A, self._dtype)

    def _buildUnitory(self, time):
        return np.asarray(-1j * self._hamiltonian * time, dtype=self._dtype)

    def _initExpMator(self, n: int, dtype=np.complex64):
        if dtype == np.complex64:
            return ExpMatComplex64(n)
        if dtype == np.complex128:
            return ExpMatComplex128(n)
        raise TypeError(f"dtype {dtype} is not supported")

    @property
    def _engine(self):
        return self._expMator._backend._engine

    def buildExpmOperator(self, time: float) -> None:
        """U = expm(-i H t), kept as a host array (FastCTQW/Operator.py:70-78)."""
        if self._edges is not None:
            import torch
            dX = self._generator_device(time)
            dU = torch.empty_like(dX)
            self._engine.run_device(dX, dU)
            self._expmMat = dU.cpu().numpy()
        else:
            self._expmMat = self._expMator.run(self._buildUnitory(time))
        self._walked = False

    def propagate(self, time: float, psi0: np.ndarray) -> np.ndarray:
        """psi = expm(-i H t) psi0 on the device; U stays there until getOperator()."""
        if self._edges is not None:
            import torch
            dX = self._generator_device(time)
            p0 = torch.from_numpy(np.ascontiguousarray(psi0, dtype=self._dtype)).cuda()
            dpsi = torch.empty_like(p0)
            self._engine.walk_device(dX, p0, dpsi)
            psi = dpsi.cpu().numpy()
            self._expmMat = None
            self._walked = False   # U of a device-built walk is not kept for getOperator
            return psi
        psi = self._engine.walk_host(self._buildUnitory(time), psi0)
        self._expmMat = None
        self._walked = True
        return psi

    def _generator_device(self, time: float, out=None):
        """X = -1j * H * t as a device tensor (built there for an edge-list operator)."""
        if self._edges is not None:
            from .device import build_generator
            return build_generator(self._n, self._edges, time, self._gamma, self._laplacian, self._dtype, out=out)
        import torch
        X = torch.from_numpy(self._buildUnitory(time))
        return X.cuda() if out is None else out.copy_(X)

    def time_curve(self, times, psi0: np.ndarray, nodes=None, method: str = "auto") -> np.ndarray:
        """Probabilities |psi(t)_v|^2 for every t of ``times`` and every node v of ``nodes``
        (all nodes when None): an array of shape (len(times), len(nodes)), the ``target_state``
        of ``Plot.timeCurve`` (FastCTQW/Plot.py:35-49).

        method "steps": the times must be the uniform grid t_k = (k + 1) dt; one exponential
        gives U(dt) and psi(t_k) = U(dt) psi(t_{k-1}) (one GEMV per time; the error grows with
        the number of steps by the rounding of U to the walk's dtype).  "batch": one walk per
        time through the grouped batch pipeline (each at the single-walk accuracy).  "auto":
        "steps" on a uniform grid, else "batch"."""
        import torch
        from .device import apply_propagator, probabilities
        times = np.asarray(times, dtype=np.float64).reshape(-1)
        K = times.shape[0]
        if K == 0:
            return np.zeros((0, self._n if nodes is None else len(nodes)))
        uniform = is_uniform_grid(times)
        if method not in ("auto", "steps", "batch"):
            raise ValueError(f"unknown method {method!r}")
        if method == "steps" and not uniform:
            raise ValueError('method="steps" needs times t_k = (k + 1) * t_0')
        p0 = torch.from_numpy(np.ascontiguousarray(psi0, dtype=self._dtype)).cuda()
        nd = None if nodes is None else torch.as_tensor(np.asarray(nodes, dtype=np.int64)).cuda()
        rows = []
        if method == "steps" or (method == "auto" and uniform):
            dX = self._generator_device(float(times[0]))
            dU = torch.empty_like(dX)
            a, b = torch.empty_like(p0), torch.empty_like(p0)
            self._engine.walk_device(dX, p0, a, dU)
            del dX
            rows.append(probabilities(a, nd))
            for _ in range(1, K):
                apply_propagator(dU, a, b)
                rows.append(probabilities(b, nd))
                a, b = b, a
            self._last_state = a
        else:
            from .batch import WalkBatch
            with WalkBatch([self._n] * K, self._dtype) as wb:
                dXs = [self._generator_device(float(t)) for t in times]
                outs = [torch.empty_like(p0) for _ in range(K)]
                wb.run_device(dXs, [p0] * K, outs)
                del dXs
            rows = [probabilities(o, nd) for o in outs]
            self._last_state = outs[-1]
        return torch.stack(rows).cpu().numpy()

    def configure(self, **kw) -> None:
        self._expMator.configure(**kw)

    def stats(self) -> dict:
        return self._expMator.stats()

    def _is_adjacency_matrix(self, A: np.ndarray) -> bool:
        if A.ndim != 2:
            print(f"Error: Matrix is not 2D. Dimensions: {A.ndim}")
            return False
        if A.shape[0] != A.shape[1]:
            print(f"Error: Matrix is not square. Shape: {A.shape}")
            return False
        if not np.array_equal(A, A.T):
            print("Error: Matrix is not symmetric (expected for undirected graph).")
            return False
        return True

    def _is_hermitian(self, hamiltonian) -> bool:
        return np.allclose(hamiltonian, hamiltonian.conj().T)

    @classmethod
    def from_networkx_graph(cls, nx_graph, gamma: float = 1, laplacian: bool = False,
                            device: str = "cuda") -> "Operator":
        import networkx as nx
        return cls(nx.to_numpy_array(nx_graph), gamma, laplacian, device)

    @classmethod
    def from_numpy_array(cls, A: np.ndarray, gamma: float = 1, laplacian: bool = False,
                         device: str = "cuda") -> "Operator":
        return cls(A, gamma, laplacian, device)

    @classmethod
    def from_num_nodes(cls, n: int, dtype=np.complex64, device: str = "cuda") -> "Operator":
        return cls(n, device=device, dtype=dtype)

    @classmethod
    def from_adjacency_list(cls, adj_list, gamma: float = 1, laplacian: bool = False, device: str = "cuda",
                            dtype=np.float32) -> "Operator":
        """Operator of the undirected graph with ``adj_list[u]`` = neighbours of u (edges are
        symmetrised; a repeated edge counts once).  ``dtype`` float32/complex64 -> complex64
        walk, float64/complex128 -> complex128, as for an adjacency matrix.  The edges live on
        the device and X = -i H t is built there (the reference declares this constructor but
        leaves it empty, FastCTQW/Operator.py:115-117)."""
        from .device import edges_from_adjacency_list
        return cls._from_edges(len(adj_list), edges_from_adjacency_list(adj_list), gamma, laplacian, device, dtype)

    @classmethod
    def _from_edges(cls, n: int, edges: np.ndarray, gamma: float, laplacian: bool, device: str,
                    dtype) -> "Operator":
        import torch
        op = cls(int(n), device=device, dtype=cls._dtype_for(np.zeros(0, dtype=dtype)))
        op._gamma = gamma
        op._laplacian = laplacian
        e = np.ascontiguousarray(edges, dtype=np.int64).reshape(-1, 2)
        if e.size and (e.min() < 0 or e.max() >= n):
            raise ValueError("an edge endpoint is outside 0..n-1")
        op._edges = torch.from_numpy(e).cuda()
        op._hamiltonian = None
        return op

    def reset_numpy_array(self, A: np.ndarray, gamma: float = 1, laplacian: bool = False):
        self._dtype = self._dtype_for(A)
        self._gamma = gamma
        self._laplacian = laplacian
        self._hamiltonian = self._buildHamiltonian(A, gamma)
        if not self._is_hermitian(self._hamiltonian):
            raise ValueError("_hamiltonian is not a hamiltonian matrix")
        if A.shape[0] != self._n or self._expMator._backend._engine.dtype != np.dtype(self._dtype):
            self._expMator.free()
            self._n = A.shape[0]
            self._expMator = self._initExpMator(self._n, self._dtype)
        self._expmMat = None
        self._walked = False

    def reset_networkx_graph(self, nx_graph, gamma: float = 1, laplacian: bool = False):
        import networkx as nx
        self.reset_numpy_array(nx.to_numpy_array(nx_graph), gamma, laplacian)

    def setHamiltonian(self, hamiltonian: NDArray):
        self._hamiltonian = hamiltonian

    def setexpmOperator(self, newexpmMat):
        self._expmMat = newexpmMat
        self._walked = False

    def getOperator(self):
        if self._expmMat is None and self._walked:
            self._expmMat = self._expMator._backend._engine.fetch_u()
        return self._expmMat
