"""Quantum state container, mirroring FastCTQW/State.py:4-59.

Amplitudes are a 1-D complex64 vector (State.py:31, :39, :45); a state whose squared norm
is off by more than 1e-5 only triggers a warning, as in the reference (:14-25), while a
non-1-D input is rejected with ``ValueError``.
"""
from __future__ import annotations

import warnings

import numpy as np


class State:
    def __init__(self, initState: np.ndarray):
        if not self._isState(initState):
            raise ValueError("initState is not a quantum state")
        self._state = initState

    def _isState(self, state: np.ndarray, tol: float = 1e-5) -> bool:
        state = np.asarray(state)
        if state.ndim != 1:
            warnings.warn(f"input is not a 1-D array (ndim = {state.ndim})")
            return False
        s = float(np.sum(np.abs(state) ** 2))
        if not np.isclose(s, 1.0, atol=tol):
            warnings.warn(f"state is not normalised: sum |amp|^2 = {s}, expected 1.0")
        return True

    @classmethod
    def getUniformSuperposition(cls, n: int) -> "State":
        return cls(np.full(n, 1.0 / np.sqrt(n), dtype=np.complex64))

    @classmethod
    def getSingleNodeState(cls, n: int, m: int) -> "State":
        s = np.zeros(n, dtype=np.complex64)
        s[m] = 1.0
        return cls(s)

    @classmethod
    def getLocalSuperposition(cls, n: int, markNodes: list) -> "State":
        s = np.zeros(n, dtype=np.complex64)
        for i in markNodes:
            s[i] = 1.0
        return cls(s / np.linalg.norm(s))

    def getProbabilities(self) -> np.ndarray:
        return np.abs(self._state) ** 2

    def setState(self, initState: np.ndarray) -> None:
        if not self._isState(initState):
            raise ValueError("initState is not a quantum state")
        self._state = initState

    def getState(self) -> np.ndarray:
        return self._state
