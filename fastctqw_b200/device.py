"""Device-side set-up and read-out of a walk (``fx_build_generator``, ``fx_check_hermitian``,
``fx_apply_propagator``, ``fx_probabilities``): the O(N^2) steps that the reference ran on the
host in numpy, done where the matrices live.

* ``build_generator``: X = -1j * H * t of an undirected graph given by its edges, H = -gamma A
  or -gamma (D - A) (FastCTQW/Operator.py:49-56), bit for bit what numpy computes from
  ``nx.to_numpy_array`` in the same dtype.
* ``is_hermitian``: ``np.allclose(H, H^H)`` (FastCTQW/Operator.py:92-103) in one pass, or the
  skew-Hermitian test of X = -iHt.
* ``apply_propagator``: psi_out = U psi_in (the GEMV of Ctqw.runWalk, FastCTQW/Ctqw.py:90-94).
* ``probabilities``: |psi|^2 of all or of marked nodes (FastCTQW/State.py:50-51), in float64.

Tensors are torch CUDA tensors; they are handed to the library as raw pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from ._native import lib

_C_OF = {"complex64": _native.DTYPE_CODE[np.dtype(np.complex64)],
         "complex128": _native.DTYPE_CODE[np.dtype(np.complex128)],
         "float32": _native.DTYPE_CODE[np.dtype(np.float32)],
         "float64": _native.DTYPE_CODE[np.dtype(np.float64)]}


def _code(t) -> int:
    name = str(t.dtype).replace("torch.", "")
    if name not in _C_OF:
        raise TypeError(f"unsupported dtype {t.dtype}")
    return _C_OF[name]


def _check(rc: int) -> None:
    if rc == _native.OK:
        return
    msg = lib().fx_graph_error()
    msg = msg.decode() if msg else f"error code {rc}"
    try:
        _native.check(rc)
    except Exception as e:  # noqa: BLE001 - re-raise the mapped type with the library message
        raise type(e)(msg) from None


def _stream(stream) -> int:
    return _native.Engine._stream(stream)


def edges_from_adjacency_list(adj_list) -> np.ndarray:
    """(m, 2) int64 edges of an adjacency list: ``adj_list[u]`` holds the neighbours of u."""
    pairs = [(u, int(v)) for u, nbrs in enumerate(adj_list) for v in nbrs]
    return np.asarray(pairs, dtype=np.int64).reshape(-1, 2)


def edges_from_networkx(graph) -> tuple[int, np.ndarray]:
    """(n, edges) of a networkx graph in the node order of ``nx.to_numpy_array``."""
    index = {v: i for i, v in enumerate(graph.nodes())}
    e = np.asarray([(index[u], index[v]) for u, v in graph.edges()], dtype=np.int64).reshape(-1, 2)
    return graph.number_of_nodes(), e


def build_generator(n: int, edges, t: float, gamma: float = 1.0, laplacian: bool = False,
                    dtype=np.complex64, out=None, stream=None):
    """X = -1j * H * t (n x n, on the device) from int64 edges (a device tensor of shape (m, 2),
    or a host array, copied over)."""
    import torch
    tdt = {np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128}.get(np.dtype(dtype))
    if tdt is None:
        raise TypeError("X is complex64 or complex128")
    if not isinstance(edges, torch.Tensor):
        edges = torch.as_tensor(np.ascontiguousarray(edges, dtype=np.int64).reshape(-1, 2))
    edges = edges.to(device="cuda", dtype=torch.int64).contiguous()
    if out is None:
        out = torch.empty((n, n), dtype=tdt, device="cuda")
    if out.shape != (n, n) or out.dtype != tdt or not out.is_contiguous():
        raise ValueError("out must be a contiguous n x n tensor of the walk's dtype")
    m = edges.shape[0]
    _check(lib().fx_build_generator(int(n), edges.data_ptr() if m else None, int(m), float(gamma),
                                    int(bool(laplacian)), float(t), _code(out), out.data_ptr(), _stream(stream)))
    return out


def is_hermitian(H, rtol: float = 1e-5, atol: float = 1e-8, skew: bool = False, stream=None) -> bool:
    """``np.allclose(H, H.conj().T, rtol, atol)`` for a square device tensor; with ``skew`` the
    test against ``-H.conj().T`` (the form of a walk's X = -iHt)."""
    H = H.contiguous()
    if H.dim() != 2 or H.shape[0] != H.shape[1]:
        raise ValueError("H must be square")
    r = ctypes.c_int32(0)
    _check(lib().fx_check_hermitian(int(H.shape[0]), _code(H), H.data_ptr(), float(rtol), float(atol),
                                    int(bool(skew)), ctypes.byref(r), _stream(stream)))
    return bool(r.value)


def apply_propagator(U, psi_in, psi_out=None, stream=None):
    """psi_out = U psi_in on the device (complex64 or complex128, FP64 accumulation)."""
    import torch
    n = U.shape[0]
    if U.shape != (n, n) or psi_in.shape != (n,) or U.dtype != psi_in.dtype:
        raise ValueError("U must be n x n and psi_in of length n, of one dtype")
    if psi_out is None:
        psi_out = torch.empty_like(psi_in)
    Uc, xc = U.contiguous(), psi_in.contiguous()   # held until the call has been issued
    _check(lib().fx_apply_propagator(int(n), _code(U), Uc.data_ptr(), xc.data_ptr(), psi_out.data_ptr(),
                                      _stream(stream)))
    return psi_out


def probabilities(psi, nodes=None, out=None, stream=None):
    """|psi_i|^2 (float64, on the device) for every node, or for the listed nodes (NaN for a
    node outside the state)."""
    import torch
    n = psi.shape[0]
    if nodes is not None and not isinstance(nodes, torch.Tensor):
        nodes = torch.as_tensor(np.asarray(nodes, dtype=np.int64))
    if nodes is not None:
        nodes = nodes.to(device="cuda", dtype=torch.int64).contiguous()
    count = n if nodes is None else nodes.shape[0]
    if out is None:
        out = torch.empty(count, dtype=torch.float64, device="cuda")
    if count:
        psi = psi.contiguous()
        _check(lib().fx_probabilities(int(n), _code(psi), psi.data_ptr(),
                                      nodes.data_ptr() if nodes is not None else None, int(count),
                                      out.data_ptr(), _stream(stream)))
    return out
