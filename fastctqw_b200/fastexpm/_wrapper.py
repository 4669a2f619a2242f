"""Python drop-in for ``FastCTQW.fastexpm`` (FastCTQW/fastexpm/_wrapper.py:9-130).

Same four classes and the same behaviour: ``run(A)`` raises ``TypeError`` for a
non-ndarray and ``ValueError`` for a shape other than (N, N) (:29-35), the objects are
context managers whose ``__exit__`` frees the device workspace, warns if that fails and
never swallows the exception in flight (:15-27).
"""
from __future__ import annotations

import warnings

import numpy as np

from . import _fastexpm_core


class _ExpMat:
    _core = None

    def __init__(self, N: int):
        self.N = N
        self._backend = self._core(N)

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_val, exc_tb):
        try:
            self.free()
        except Exception as cleanup_error:  # noqa: BLE001 - mirrored behaviour
            warnings.warn(f"[fastexpm] Failed to free resources in __exit__: {cleanup_error}")
        return False

    def run(self, A) -> np.ndarray:
        if not isinstance(A, np.ndarray):
            raise TypeError("Input must be a NumPy array.")
        if A.shape != (self.N, self.N):
            raise ValueError(f"Input matrix must have shape ({self.N}, {self.N}).")
        return self._backend.run(A).reshape(self.N, self.N)

    def run_device(self, dA, dU, stream=None) -> None:
        """Device-resident variant: torch CUDA tensors (or raw pointers) in and out."""
        self._backend.run_device(dA, dU, stream)

    def configure(self, **kw) -> None:
        """Arithmetic options: form ('plain' | 'mixed' | 'simt'), shift, structure, ..."""
        self._backend.configure(**kw)

    def stats(self) -> dict:
        """(m, s), norms, form and device time of the last run."""
        return self._backend.stats()

    def free(self):
        self._backend.free()


class ExpMatFloat32(_ExpMat):
    _core = _fastexpm_core.ExpMatFloat32


class ExpMatFloat64(_ExpMat):
    _core = _fastexpm_core.ExpMatFloat64


class ExpMatComplex64(_ExpMat):
    _core = _fastexpm_core.ExpMatComplex64


class ExpMatComplex128(_ExpMat):
    _core = _fastexpm_core.ExpMatComplex128
