"""Batched walks: many independent walks of uneven sizes through grouped device launches.

The reference runs one walk at a time (``Ctqw.runWalk``, FastCTQW/Ctqw.py:90-94, one
``MatrixExpCalculator`` per matrix size, include/MatrixExpCalculator.h:17-103).
:class:`WalkBatch` runs ``psi_w = expm(X_w) psi0_w`` for a whole list of walks at once through
the C ABI's ``fx_batch_*`` entry points: every phase of the scaling-and-squaring pipeline is
one grouped launch over all walks, and everything after the (m, s) selection is replayed as
one CUDA graph.  The generators must be walk generators ``X = -1j * H * t`` with a real
symmetric H (``ValueError`` otherwise); the dtype is complex64 or complex128.

    >>> b = WalkBatch([A.shape[0] for A in adjs])
    >>> psis = b.run([walk_generator(A, t) for A, t in zip(adjs, ts)], psi0s)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from ._native import check, lib

OPT_GRAPH, OPT_TIMEOUT_MS, OPT_FORCE_M, OPT_SELECTOR, OPT_ANALYZE_ONLY, OPT_DIAG_SPLIT = 0, 1, 2, 3, 4, 5
OPT_AUTOTUNE, OPT_TILE_GROUP, OPT_TILE_ORDER, OPT_SAMPLE_WALKS = 6, 7, 8, 9
OPT_FORM, OPT_SQ_N4, OPT_SQ_N3, OPT_DRIFT, OPT_PADE_SLICES, OPT_NEWTON_SLICES, OPT_SOLVE = 10, 11, 12, 13, 14, 15, 16
OPT_APPROX = 17
OUTCOMES = {0: "plain", 1: "certified", 2: "learned", 3: "estimated",
            -1: "learned rejected by the bound, plain (m, s) kept",
            -2: "failed an a-posteriori check, redone with the plain (m, s)", 4: "forced (m, s)",
            5: "Chebyshev polynomial"}


def _check(rc: int, h) -> None:
    if rc == _native.OK:
        return
    msg = lib().fx_batch_last_error(h)
    msg = msg.decode() if msg else f"error code {rc}"
    try:
        check(rc)
    except Exception as e:  # noqa: BLE001 - re-raise the mapped type with the batch message
        raise type(e)(msg) from None


def walk_generator(A: np.ndarray, t: float, gamma: float = 1.0, laplacian: bool = False,
                   dtype=np.complex64) -> np.ndarray:
    """X = -1j * H * t with H = -gamma A or -gamma (D - A) (FastCTQW/Operator.py:49-56)."""
    A = np.asarray(A, dtype=np.float64)
    H = -gamma * ((np.diag(A.sum(axis=1)) - A) if laplacian else A)
    return np.asarray(-1j * H * t, dtype=dtype)


class WalkBatch:
    """Owner of one ``fx_batch`` handle: device workspace for walks of sizes ``ns``."""

    def __init__(self, ns, dtype=np.complex64, graph: bool = True, selector: str = "plain",
                 analyze_only: bool = False, diag_split: int = 7, autotune: bool = False,
                 form: str = "plain", sq_n4: int | None = None, sq_n3: int | None = None,
                 drift: bool = False, pade_slices: int | None = None,
                 newton_slices: int | None = None, solve: str = "auto", approx: str = "pade") -> None:
        self.ns = [int(n) for n in ns]
        self.dtype = np.dtype(dtype)
        if self.dtype not in (np.dtype(np.complex64), np.dtype(np.complex128)):
            raise TypeError("batched walks are complex64 or complex128")
        arr = (ctypes.c_int64 * len(self.ns))(*self.ns)
        h = ctypes.c_void_p()
        _check(lib().fx_batch_create(len(self.ns), arr, _native.DTYPE_CODE[self.dtype], ctypes.byref(h)), None)
        self._h = h
        if not graph:
            self.set_option(OPT_GRAPH, 0)
        if selector != "plain":
            self.set_option(OPT_SELECTOR, _native.SELECTORS[selector])
        if analyze_only:
            self.set_option(OPT_ANALYZE_ONLY, 1)
        if int(diag_split) != 7:
            self.set_option(OPT_DIAG_SPLIT, int(diag_split))
        if autotune:
            self.set_option(OPT_AUTOTUNE, 1)
        if sq_n4 is not None:
            self.set_option(OPT_SQ_N4, sq_n4)
        if sq_n3 is not None:
            self.set_option(OPT_SQ_N3, sq_n3)
        if pade_slices is not None:
            self.set_option(OPT_PADE_SLICES, pade_slices)
        if newton_slices is not None:
            self.set_option(OPT_NEWTON_SLICES, newton_slices)
        if solve != "auto":
            self.set_option(OPT_SOLVE, _native.SOLVES[solve])
        if approx != "pade":
            if approx not in _native.APPROXES:
                raise ValueError(f"approx must be one of {sorted(_native.APPROXES)}")
            self.set_option(OPT_APPROX, _native.APPROXES[approx])
        if form != "plain":
            if form != "mixed":
                raise ValueError("batched walks take form 'plain' or 'mixed'")
            self.set_option(OPT_FORM, _native.FORM_MIXED)
        if drift:
            self.set_option(OPT_DRIFT, 1)

    def force_selection(self, m=None, s=None) -> None:
        """Per-walk forced (m, s) for the next runs (m[w] <= 0: the walk's own selection); no
        arguments clears."""
        if m is None:
            _check(lib().fx_batch_force_selection(self._h, None, None), self._h)
            return
        n = len(self.ns)
        mm = (ctypes.c_int32 * n)(*[int(x) for x in m])
        ss = (ctypes.c_int32 * n)(*[int(x) for x in s])
        _check(lib().fx_batch_force_selection(self._h, mm, ss), self._h)

    def spectral(self) -> dict:
        """Per walk: Lanczos spectral-radius estimate and rigorous bound of the last run."""
        n = len(self.ns)
        a = (ctypes.c_double * n)()
        b = (ctypes.c_double * n)()
        _check(lib().fx_batch_spectral(self._h, a, b), self._h)
        return {"lanczos": np.array(a[:]), "upper_bound": np.array(b[:])}

    def drift(self, w: int) -> list:
        """||U_k^H U_k - I||_F / sqrt(n) after every squaring of walk w in the last run (needs
        drift=True)."""
        cnt = ctypes.c_int32()
        buf = (ctypes.c_double * 64)()
        _check(lib().fx_batch_drift(self._h, int(w), buf, 64, ctypes.byref(cnt)), self._h)
        return list(buf[:min(cnt.value, 64)])

    def set_option(self, key: int, value: float) -> None:
        _check(lib().fx_batch_set_option(self._h, int(key), float(value)), self._h)

    def _ptrs(self, xs):
        return (ctypes.c_void_p * len(xs))(*[ctypes.c_void_p(x) for x in xs])

    def run(self, Xs, psi0s=None) -> list[np.ndarray]:
        """psi_w = expm(X_w) psi0_w for host ndarrays; returns a list of new arrays."""
        if len(Xs) != len(self.ns) or (psi0s is not None and len(psi0s) != len(self.ns)):
            raise ValueError(f"expected {len(self.ns)} generators and states")
        xs, p0, p1 = [], [], []
        if psi0s is None:
            psi0s = [np.full(n, 1.0 / np.sqrt(n), dtype=self.dtype) for n in self.ns]
        for X, p, n in zip(Xs, psi0s, self.ns):
            X = np.ascontiguousarray(X, dtype=self.dtype)
            if X.shape != (n, n):
                raise ValueError(f"Input matrix must have shape ({n}, {n}).")
            p = np.ascontiguousarray(p, dtype=self.dtype).reshape(-1)
            if p.shape != (n,):
                raise ValueError(f"state must have length {n}")
            xs.append(X)
            p0.append(p)
            p1.append(np.empty(n, dtype=self.dtype))
        _check(lib().fx_batch_walk_host(self._h, self._ptrs([x.ctypes.data for x in xs]),
                                        self._ptrs([p.ctypes.data for p in p0]),
                                        self._ptrs([p.ctypes.data for p in p1])), self._h)
        return p1

    def run_device(self, dXs, dpsi0s, dpsis, stream=None) -> None:
        """The same on device buffers (torch CUDA tensors or raw pointers)."""
        P = _native.Engine._ptr
        s = _native.Engine._stream(stream)
        _check(lib().fx_batch_walk_device(self._h, self._ptrs([P(x) for x in dXs]),
                                          self._ptrs([P(x) for x in dpsi0s]),
                                          self._ptrs([P(x) for x in dpsis]), s), self._h)

    def selection(self) -> tuple[np.ndarray, np.ndarray]:
        """(m, s) of every walk in the last run."""
        m = (ctypes.c_int32 * len(self.ns))()
        s = (ctypes.c_int32 * len(self.ns))()
        _check(lib().fx_batch_selection(self._h, m, s), self._h)
        return np.array(m[:], dtype=np.int32), np.array(s[:], dtype=np.int32)

    def sample_check(self) -> dict:
        """The last run's sampled comparison with the plain method: walks re-run (0 when no
        walk took a non-plain (m, s), -1 when skipped for a batch of one walk), largest
        infidelity between the two states."""
        c, m = ctypes.c_int32(), ctypes.c_double()
        _check(lib().fx_batch_sample_check(self._h, ctypes.byref(c), ctypes.byref(m)), self._h)
        return {"sampled": c.value, "max_infidelity": m.value}

    def schedule(self) -> dict:
        """Schedule of the post-selection products (tile group, tile order) and, after an
        autotuned run, the candidates tried with their times."""
        g, o, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        t = (ctypes.c_double * 48)()
        _check(lib().fx_batch_schedule(self._h, ctypes.byref(g), ctypes.byref(o), t, ctypes.byref(n)), self._h)
        return {"tile_group": g.value, "tile_order": o.value,
                "tuned": [(int(t[3 * i]), int(t[3 * i + 1]), t[3 * i + 2]) for i in range(n.value)]}

    def set_schedule(self, tile_group: int, tile_order: int) -> None:
        self.set_option(OPT_TILE_GROUP, tile_group)
        self.set_option(OPT_TILE_ORDER, tile_order)

    def details(self) -> dict:
        """Per walk of the last run: selector features (n x 8), the Al-Mohy & Higham (m, s),
        the certified (m, s) and the selection outcome (see OUTCOMES)."""
        W = len(self.ns)
        f = (ctypes.c_double * (8 * W))()
        arr = [(ctypes.c_int32 * W)() for _ in range(5)]
        _check(lib().fx_batch_details(self._h, f, *arr), self._h)
        out = {"features": np.array(f[:], dtype=np.float64).reshape(W, 8)}
        for name, a in zip(("plain_m", "plain_s", "cert_m", "cert_s", "outcome"), arr):
            out[name] = np.array(a[:], dtype=np.int32)
        return out

    def info(self) -> dict:
        """Device time (ms), algorithmic flops and kernel launches of the last run."""
        ms, fl, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32()
        _check(lib().fx_batch_info(self._h, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(nl)), self._h)
        return {"ms": ms.value, "flops": fl.value, "launches": nl.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fx_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
