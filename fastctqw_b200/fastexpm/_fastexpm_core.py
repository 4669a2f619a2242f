"""Native expm classes, the counterpart of the reference's pybind11 module ``_fastexpm_core``
(src/main.cu:8-64): ``ExpMatFloat32``, ``ExpMatFloat64``, ``ExpMatComplex64`` and
``ExpMatComplex128`` with ``__init__(n)`` (allocates the device workspace), ``run(arr_a)``
and ``free()``.  Each class owns one handle of the C ABI (include/fastctqw_b200.h) through
:class:`fastctqw_b200._native.Engine`.

As with pybind11's ``py::array_t<T>`` (which force-casts), ``run`` converts its argument to
the class's element type.
"""
from __future__ import annotations

import numpy as np

from .._native import Engine


class _ExpMatCore:
    _dtype = None

    def __init__(self, n: int):
        self._engine = Engine(int(n), self._dtype)
        self.n = int(n)

    def run(self, arr_a) -> np.ndarray:
        """expm(arr_a) for an (n, n) array; returns a new (n, n) array."""
        return self._engine.run_host(arr_a)

    def run_device(self, dA, dU, stream=None) -> None:
        """expm on device buffers (torch tensors or raw pointers), ordered on ``stream``."""
        self._engine.run_device(dA, dU, stream)

    def configure(self, **kw) -> None:
        self._engine.configure(**kw)

    def stats(self) -> dict:
        return self._engine.stats()

    def getN(self) -> int:  # MatrixExpCalculator<T>::getN (include/MatrixExpCalculator.h:41)
        return self.n

    def free(self) -> None:
        self._engine.free()


class ExpMatFloat32(_ExpMatCore):
    _dtype = np.float32


class ExpMatFloat64(_ExpMatCore):
    _dtype = np.float64


class ExpMatComplex64(_ExpMatCore):
    _dtype = np.complex64


class ExpMatComplex128(_ExpMatCore):
    _dtype = np.complex128
