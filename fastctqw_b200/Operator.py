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
  parameters (the reference mixed them up, :118-120, :144-146).
"""
from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

from .fastexpm import ExpMatComplex64, ExpMatComplex128


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

    def buildExpmOperator(self, time: float) -> None:
        """U = expm(-i H t), kept as a host array (FastCTQW/Operator.py:70-78)."""
        self._expmMat = self._expMator.run(self._buildUnitory(time))
        self._walked = False

    def propagate(self, time: float, psi0: np.ndarray) -> np.ndarray:
        """psi = expm(-i H t) psi0 on the device; U stays there until getOperator()."""
        psi = self._expMator._backend._engine.walk_host(self._buildUnitory(time), psi0)
        self._expmMat = None
        self._walked = True
        return psi

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
