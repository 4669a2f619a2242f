"""ctypes binding of the C ABI in ``include/fastctqw_b200.h``.

The shared library ``lib/libfastctqw_b200.so`` (built by ``python -m fastctqw_b200.build``)
is the only compute path.  There is no CPU fallback: if the library or an sm_100 device
is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libfastctqw_b200.so")

F32, F64, C64, C128 = 0, 1, 2, 3
DTYPE_CODE = {np.dtype(np.float32): F32, np.dtype(np.float64): F64,
              np.dtype(np.complex64): C64, np.dtype(np.complex128): C128}
CODE_DTYPE = {v: k for k, v in DTYPE_CODE.items()}

FORM_PLAIN, FORM_MIXED, FORM_SIMT, FORM_FP64 = 0, 1, 2, 3
FORMS = {"plain": FORM_PLAIN, "mixed": FORM_MIXED, "simt": FORM_SIMT, "fp64": FORM_FP64}
(OPT_FORM, OPT_SHIFT, OPT_STRUCTURE, OPT_FORCE_S, OPT_FORCE_M, OPT_TIMEOUT_MS, OPT_IPE, OPT_REFINE,
 OPT_DEBUG_STAGE, OPT_PROFILE, OPT_SELECTOR, OPT_INJECT_STALL, OPT_SQ_N4, OPT_SQ_N3, OPT_DRIFT,
 OPT_PADE_SLICES, OPT_NEWTON_SLICES, OPT_SOLVE, OPT_APPROX) = range(19)
SOLVES = {"auto": 0, "cholesky": 1, "newton": 2}
APPROXES = {"pade": 0, "chebyshev": 1}
SELECTORS = {"plain": 0, "certified": 1, "learned": 2, "estimated": 3}

OK, ERR_TYPE, ERR_VALUE, ERR_NOMEM, ERR_CUDA, ERR_TIMEOUT, ERR_NONFINITE, ERR_SINGULAR, ERR_NODEV, ERR_FREED = range(10)


class FxStats(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int32), ("s", ctypes.c_int32), ("form", ctypes.c_int32),
                ("structured", ctypes.c_int32), ("rank1_shift", ctypes.c_int32),
                ("symmetric", ctypes.c_int32), ("gemm_launches", ctypes.c_int32),
                ("launches", ctypes.c_int32), ("solver", ctypes.c_int32),
                ("degree", ctypes.c_int32), ("norm1", ctypes.c_double),
                ("d", ctypes.c_double * 5), ("ms_total", ctypes.c_double),
                ("flops", ctypes.c_double), ("prod_ms", ctypes.c_double),
                ("prod_ops", ctypes.c_double), ("prod_flops", ctypes.c_double),
                ("prod_launches", ctypes.c_int32), ("reserved2", ctypes.c_int32),
                ("selector", ctypes.c_int32), ("sel_outcome", ctypes.c_int32),
                ("plain_m", ctypes.c_int32), ("plain_s", ctypes.c_int32)]

    def as_dict(self) -> dict:
        out = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("d", "reserved2")}
        out["d4"], out["d6"], out["d8"], out["d10"], out["log2_abs27"] = list(self.d)
        return out


_lib = None
_lock = threading.Lock()

# (name, argtypes) of every symbol declared in include/fastctqw_b200.h
SIGNATURES = {
    "fx_create": [ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "fx_destroy": [ctypes.c_void_p],
    "fx_free": [ctypes.c_void_p],
    "fx_get_n": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)],
    "fx_set_option": [ctypes.c_void_p, ctypes.c_int, ctypes.c_double],
    "fx_get_stats": [ctypes.c_void_p, ctypes.POINTER(FxStats)],
    "fx_spectral_radius": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
    "fx_batch_force_selection": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
    "fx_batch_spectral": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
    "fx_chebyshev_plan": [ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_int32),
                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                          ctypes.POINTER(ctypes.c_int32)],
    "fx_unitarity_drift": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int32,
                           ctypes.POINTER(ctypes.c_int32)],
    "fx_batch_drift": [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double), ctypes.c_int32,
                       ctypes.POINTER(ctypes.c_int32)],
    "fx_product_profile": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)],
    "fx_last_error": [ctypes.c_void_p],
    "fx_run_host": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fx_run_device": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fx_walk_device": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_void_p],
    "fx_walk_host": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fx_fetch_u": [ctypes.c_void_p, ctypes.c_void_p],
    "fx_product_f32": [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                       ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                       ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_int64,
                       ctypes.c_float, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    "fx_product_error": [],
    "fx_slice_rows_f64": [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                          ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fx_tensor_peak": [ctypes.c_int, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                       ctypes.POINTER(ctypes.c_double), ctypes.c_void_p],
    "fx_build_generator": [ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int,
                           ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    "fx_check_hermitian": [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                           ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p],
    "fx_apply_propagator": [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p],
    "fx_probabilities": [ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                         ctypes.c_void_p, ctypes.c_void_p],
    "fx_graph_error": [],
    "fx_batch_sample_check": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)],
    "fx_batch_schedule": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)],
    "fx_product_f32_noalloc": [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                               ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                               ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_int64,
                               ctypes.c_float, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    "fx_batch_create": [ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64), ctypes.c_int,
                        ctypes.POINTER(ctypes.c_void_p)],
    "fx_batch_destroy": [ctypes.c_void_p],
    "fx_batch_set_option": [ctypes.c_void_p, ctypes.c_int, ctypes.c_double],
    "fx_batch_walk_device": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                             ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                             ctypes.c_void_p],
    "fx_batch_walk_host": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                           ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)],
    "fx_batch_selection": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                           ctypes.POINTER(ctypes.c_int32)],
    "fx_batch_info": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)],
    "fx_batch_last_error": [ctypes.c_void_p],
    "fx_batch_details": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32),
                         ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                         ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
    "fx_selector_set_weights": [ctypes.POINTER(ctypes.c_float), ctypes.c_int64],
    "fx_mlp_param_count": [],
    "fx_mlp_infer": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p],
    "fx_mlp_loss_grad": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                         ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "fx_mlp_train": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                     ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                     ctypes.POINTER(ctypes.c_float), ctypes.c_void_p],
    "fx_mlp_error": [],
    "fx_gpu_memory_gb": [],
    "fx_device_ok": [],
    "fx_version": [],
}
RESTYPES = {"fx_last_error": ctypes.c_char_p, "fx_version": ctypes.c_char_p,
            "fx_batch_last_error": ctypes.c_char_p, "fx_mlp_error": ctypes.c_char_p,
            "fx_product_error": ctypes.c_char_p,
            "fx_graph_error": ctypes.c_char_p,
            "fx_gpu_memory_gb": ctypes.c_double}


def lib() -> ctypes.CDLL:
    """Load the native library (once).  Raises ImportError when it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"native library missing: {LIB_PATH} (build it with python -m fastctqw_b200.build)")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in SIGNATURES.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = RESTYPES.get(name, ctypes.c_int)
            _lib = L
    return _lib


def last_error(h=None) -> str:
    msg = lib().fx_last_error(h)
    return msg.decode() if msg else ""


def check(rc: int, h=None) -> None:
    if rc == OK:
        return
    msg = last_error(h) or f"error code {rc}"
    if rc == ERR_TYPE:
        raise TypeError(msg)
    if rc in (ERR_VALUE, ERR_NONFINITE):
        raise ValueError(msg)
    if rc == ERR_NOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def product_f32(form: str, A, Bt, alpha=1.0, beta=0.0, C=None, gamma=0.0, D=None):
    """D = alpha A Bt^T + beta C + gamma I with torch CUDA float32 tensors (diagnostic)."""
    import torch
    M, K = A.shape
    N = Bt.shape[0]
    if D is None:
        D = torch.empty((M, N), device=A.device, dtype=torch.float32)
    rc = lib().fx_product_f32(FORMS[form], M, N, K, A.data_ptr(), A.stride(0), Bt.data_ptr(),
                              Bt.stride(0), alpha, beta, C.data_ptr() if C is not None else None,
                              C.stride(0) if C is not None else 0, gamma, D.data_ptr(), D.stride(0),
                              torch.cuda.current_stream().cuda_stream)
    if rc != OK:
        raise RuntimeError(lib().fx_product_error().decode())
    return D


def slice_rows(re, im=None, S: int = 5, kind: int = 1, split_diag: bool = False, neg: bool = False) -> dict:
    """The product kernels' int8 slicer on torch CUDA float64 rows (diagnostic, fx_slice_rows_f64):
    digits (S, rows, K) of re (and of im, -im), row exponents, split-off diagonal."""
    import torch
    rows, K = re.shape
    if im is not None and (im.shape != re.shape or im.stride() != re.stride()):
        raise ValueError("slice_rows: re and im need the same shape and strides")
    ldo = (K + 15) // 16 * 16
    out = torch.zeros((3 * S, rows, ldo), dtype=torch.int8, device=re.device)
    exps = torch.zeros(rows, dtype=torch.int32, device=re.device)
    dg = torch.zeros(rows, dtype=torch.float64, device=re.device) if split_diag else None
    rc = lib().fx_slice_rows_f64(kind, S, re.data_ptr(), im.data_ptr() if im is not None else None, re.stride(0),
                                 rows, K, int(split_diag), int(neg), out.data_ptr(), ldo, exps.data_ptr(),
                                 dg.data_ptr() if dg is not None else None,
                                 torch.cuda.current_stream().cuda_stream)
    if rc != OK:
        raise RuntimeError(lib().fx_product_error().decode())
    return {"re": out[:S, :, :K], "im": out[S:2 * S, :, :K], "neg_im": out[2 * S:, :, :K], "exp": exps, "dg": dg}


def tensor_peak(kind: str = "int8", iters: int = 50000, reps: int = 5, stream=None) -> dict:
    """Measured dense tensor-core rate (fx_tensor_peak): the median of `reps` launches, in
    tera-ops per second (2 M N K per instruction)."""
    k = {"int8": 0, "bf16": 1}[kind]
    tops, ms = ctypes.c_double(), ctypes.c_double()
    vals = []
    for _ in range(reps + 1):   # the first launch warms up
        rc = lib().fx_tensor_peak(k, int(iters), ctypes.byref(tops), ctypes.byref(ms), stream)
        if rc != OK:
            raise RuntimeError(lib().fx_product_error().decode())
        vals.append((tops.value, ms.value))
    vals = sorted(vals[1:])
    return {"tops": vals[len(vals) // 2][0], "ms": vals[len(vals) // 2][1], "reps": reps,
            "all_tops": [round(v[0], 1) for v in vals]}


def chebyshev_plan(rho: float, tol: float = 1e-6) -> dict:
    """The Chebyshev approximant's plan for a spectral bound rho (fx_chebyshev_plan; host
    arithmetic, no device): squarings s, degree, baby steps and matrix products of the walk."""
    s, d, m, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    rc = lib().fx_chebyshev_plan(float(rho), float(tol), ctypes.byref(s), ctypes.byref(d),
                                 ctypes.byref(m), ctypes.byref(c))
    if rc != OK:
        msg = lib().fx_batch_last_error(None)
        raise ValueError(msg.decode() if msg else f"error code {rc}")
    return {"s": s.value, "degree": d.value, "baby": m.value, "cost": c.value}


def device_ok() -> bool:
    return bool(lib().fx_device_ok())


class Engine:
    """Owner of one native fx_engine handle (workspace for n x n matrices of one dtype)."""

    def __init__(self, n: int, dtype) -> None:
        self.dtype = np.dtype(dtype)
        if self.dtype not in DTYPE_CODE:
            raise TypeError(f"unsupported dtype {self.dtype}")
        if int(n) < 0:
            raise ValueError("n must be non-negative")
        self.n = int(n)
        h = ctypes.c_void_p()
        check(lib().fx_create(self.n, DTYPE_CODE[self.dtype], ctypes.byref(h)))
        self._h = h
        self._freed = False

    # -- options
    def set_option(self, key: int, value: float) -> None:
        check(lib().fx_set_option(self._h, int(key), float(value)), self._h)

    def configure(self, form: str | None = None, shift: int | None = None,
                  structure: bool | None = None, force_m: int | None = None,
                  force_s: int | None = None, ipe: bool | None = None,
                  timeout_ms: float | None = None, debug_stage: int | None = None,
                  profile: bool | None = None, selector: str | None = None,
                  inject_stall: int | None = None, sq_n4: int | None = None, sq_n3: int | None = None,
                  drift: bool | None = None, pade_slices: int | None = None,
                  newton_slices: int | None = None, solve: str | None = None,
                  approx: str | None = None) -> None:
        if form is not None:
            if form not in FORMS:
                raise ValueError(f"form must be one of {sorted(FORMS)}")
            self.set_option(OPT_FORM, FORMS[form])
        if shift is not None:
            self.set_option(OPT_SHIFT, shift)
        if structure is not None:
            self.set_option(OPT_STRUCTURE, int(structure))
        if force_m is not None:
            self.set_option(OPT_FORCE_M, force_m)
        if force_s is not None:
            self.set_option(OPT_FORCE_S, force_s)
        if ipe is not None:
            self.set_option(OPT_IPE, int(bool(ipe)))
        if timeout_ms is not None:
            self.set_option(OPT_TIMEOUT_MS, timeout_ms)
        if debug_stage is not None:
            self.set_option(OPT_DEBUG_STAGE, debug_stage)
        if profile is not None:
            self.set_option(OPT_PROFILE, int(bool(profile)))
        if selector is not None:
            if selector not in SELECTORS:
                raise ValueError(f"selector must be one of {sorted(SELECTORS)}")
            self.set_option(OPT_SELECTOR, SELECTORS[selector])
        if inject_stall is not None:
            self.set_option(OPT_INJECT_STALL, inject_stall)
        if sq_n4 is not None:
            self.set_option(OPT_SQ_N4, sq_n4)
        if sq_n3 is not None:
            self.set_option(OPT_SQ_N3, sq_n3)
        if drift is not None:
            self.set_option(OPT_DRIFT, int(bool(drift)))
        if pade_slices is not None:
            self.set_option(OPT_PADE_SLICES, pade_slices)
        if newton_slices is not None:
            self.set_option(OPT_NEWTON_SLICES, newton_slices)
        if solve is not None:
            if solve not in SOLVES:
                raise ValueError(f"solve must be one of {sorted(SOLVES)}")
            self.set_option(OPT_SOLVE, SOLVES[solve])
        if approx is not None:
            if approx not in APPROXES:
                raise ValueError(f"approx must be one of {sorted(APPROXES)}")
            self.set_option(OPT_APPROX, APPROXES[approx])

    def spectral_radius(self) -> dict:
        """Lanczos estimate and rigorous upper bound of the shifted generator's spectral radius
        in the last walk-generator run."""
        a, b = ctypes.c_double(), ctypes.c_double()
        check(lib().fx_spectral_radius(self._h, ctypes.byref(a), ctypes.byref(b)), self._h)
        return {"lanczos": a.value, "upper_bound": b.value}

    def unitarity_drift(self) -> list:
        """||U_k^H U_k - I||_F / sqrt(n) after every squaring k = 0..s of the last run made with
        configure(drift=True) (walk generators)."""
        cnt = ctypes.c_int32()
        buf = (ctypes.c_double * 64)()
        check(lib().fx_unitarity_drift(self._h, buf, 64, ctypes.byref(cnt)), self._h)
        return list(buf[:min(cnt.value, 64)])

    def stats(self) -> dict:
        st = FxStats()
        check(lib().fx_get_stats(self._h, ctypes.byref(st)), self._h)
        return st.as_dict()

    PRODUCT_STAGES = ("powers", "pade", "solve", "cholesky", "inverse", "triangular", "squarings",
                      "diagnostics", "newton")
    TIMELINE = ("phase1", "host_gap", "phase2", "checks")

    def product_profile(self) -> dict:
        """Per-stage product time of the last profiled walk-generator run (configure(profile=True)):
        {stage: {"launches", "ms", "ops"}}."""
        cnt = ctypes.c_int32()
        check(lib().fx_product_profile(self._h, None, None, None, 0, ctypes.byref(cnt)), self._h)
        n = cnt.value
        tags = (ctypes.c_int32 * max(n, 1))()
        ms = (ctypes.c_double * max(n, 1))()
        ops = (ctypes.c_double * max(n, 1))()
        check(lib().fx_product_profile(self._h, tags, ms, ops, n, ctypes.byref(cnt)), self._h)
        out: dict = {}
        for i in range(n):
            if tags[i] >= len(self.PRODUCT_STAGES):
                continue   # timeline records: timeline()
            d = out.setdefault(self.PRODUCT_STAGES[tags[i]], {"launches": 0, "ms": 0.0, "ops": 0.0})
            d["launches"] += 1
            d["ms"] += ms[i]
            d["ops"] += ops[i]
        self._timeline = {self.TIMELINE[tags[i] - len(self.PRODUCT_STAGES)]: ms[i]
                          for i in range(n) if tags[i] >= len(self.PRODUCT_STAGES)}
        return out

    def timeline(self) -> dict:
        """Device time of the last profiled walk-generator run by part (ms): phase 1, the gap
        between the phases, phase 2, the checks (read with product_profile)."""
        self.product_profile()
        return dict(self._timeline)

    # -- host buffers
    def _host_in(self, A) -> np.ndarray:
        A = np.ascontiguousarray(A, dtype=self.dtype)  # forcecast, like pybind11 array_t<T>
        if A.shape != (self.n, self.n):
            raise ValueError(f"Input matrix must have shape ({self.n}, {self.n}).")
        return A

    def run_host(self, A) -> np.ndarray:
        A = self._host_in(A)
        U = np.empty((self.n, self.n), dtype=self.dtype)
        check(lib().fx_run_host(self._h, A.ctypes.data, U.ctypes.data), self._h)
        return U

    def walk_host(self, A, psi0) -> np.ndarray:
        A = self._host_in(A)
        vdt = np.complex128 if self.dtype in (np.dtype(np.complex128), np.dtype(np.float64)) else np.complex64
        psi0 = np.ascontiguousarray(psi0, dtype=vdt).reshape(-1)
        if psi0.shape != (self.n,):
            raise ValueError(f"state must have length {self.n}")
        psi = np.empty(self.n, dtype=vdt)
        check(lib().fx_walk_host(self._h, A.ctypes.data, psi0.ctypes.data, psi.ctypes.data), self._h)
        return psi

    def fetch_u(self) -> np.ndarray:
        """U of the last walk_host call (it stays on the device until asked for)."""
        U = np.empty((self.n, self.n), dtype=self.dtype)
        check(lib().fx_fetch_u(self._h, U.ctypes.data), self._h)
        return U

    # -- device buffers (torch tensors or raw pointers)
    @staticmethod
    def _ptr(x) -> int:
        return x.data_ptr() if hasattr(x, "data_ptr") else int(x)

    @staticmethod
    def _stream(stream) -> int:
        if stream is None:
            try:
                import torch
                return torch.cuda.current_stream().cuda_stream
            except Exception:  # noqa: BLE001 - plain pointer callers pass their own stream
                return 0
        return int(getattr(stream, "cuda_stream", stream))

    def run_device(self, dA, dU, stream=None) -> None:
        check(lib().fx_run_device(self._h, self._ptr(dA), self._ptr(dU), self._stream(stream)), self._h)

    def walk_device(self, dA, dpsi0, dpsi, dU=None, stream=None) -> None:
        check(lib().fx_walk_device(self._h, self._ptr(dA), self._ptr(dpsi0), self._ptr(dpsi),
                                   self._ptr(dU) if dU is not None else None,
                                   self._stream(stream)), self._h)

    def free(self) -> None:
        if not self._freed:
            check(lib().fx_free(self._h), self._h)
            self._freed = True

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fx_destroy(self._h)
            self._h = None
            self._freed = True

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
