"""The allocation-free product entry point, fx_product_f32_noalloc (needs a GPU).

Callers that may not allocate device memory while they run (a memory pool that owns the
device, an allocator's own callback, a host that sizes every GPU buffer at start-up) use
fx_product_f32_noalloc instead of fx_product_f32: the same int8-slice tensor-core product, with
its scratch in a fixed array of device memory inside the library instead of a cudaMalloc per
call.  Both are called through the C ABI on the same inputs and must agree within the
complex64 tolerance the parity tests use (1e-5 relative, Frobenius); two calls in a row with
different shapes check that the shared scratch carries nothing from one call to the next.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from fastctqw_b200 import _native

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5          # complex64 tolerance of tests/test_gpu_parity.py
FORM_PLAIN = _native.FORM_PLAIN
SCRATCH_BYTES = 16 << 20


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _call(fn, M, N, K, A, Bt, alpha, beta, C, gamma, D, stream, form=None):
    args = [M, N, K, _p(A), A.stride(0), _p(Bt), Bt.stride(0), alpha, beta, _p(C),
            C.stride(0) if C is not None else 0, gamma, _p(D), D.stride(0), stream]
    return fn(form, *args) if form is not None else fn(*args)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_matches_allocating_product_twice():
    import torch
    lib = _native.lib()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    gen = torch.Generator(device="cpu").manual_seed(11)
    cases = [
        # (M, N, K, alpha, beta, gamma), one call after another on the shared array:
        (256, 384, 640, 1.0, 0.0, 0.0),        # whole 128-row tiles
        (512, 512, 1024, -0.75, 2.0, 1.5),
        (144, 208, 64, 1.25, -0.5, 0.25),      # partial tiles: clipped rows and columns, one K step
        (1408, 1408, 1408, 1.0, 1.0, -2.0),    # the largest square size the array holds
    ]
    for M, N, K, alpha, beta, gamma in cases:
        A = torch.randn(M, K, generator=gen).to(dev)
        A[::7] *= 1e-3    # rows of very different size (one exponent per row)
        Bt = torch.randn(N, K, generator=gen).to(dev)
        C = torch.randn(M, N, generator=gen).to(dev) if beta != 0.0 else None
        D_ref = torch.full((M, N), float("nan"), device=dev)
        D_new = torch.full((M, N), float("nan"), device=dev)
        rc = _call(lib.fx_product_f32, M, N, K, A, Bt, alpha, beta, C, gamma, D_ref, stream,
                   form=FORM_PLAIN)
        assert rc == _native.OK, lib.fx_product_error()
        rc = _call(lib.fx_product_f32_noalloc, M, N, K, A, Bt, alpha, beta, C, gamma, D_new, stream)
        assert rc == _native.OK, lib.fx_product_error()
        torch.cuda.synchronize()
        ref = D_ref.double().cpu().numpy()
        new = D_new.double().cpu().numpy()
        assert np.isfinite(new).all()
        assert _rel(new, ref) <= REL_TOL, (M, N, K, _rel(new, ref))
        # and both against an FP64 matmul of the same FP32 inputs
        exact = alpha * (A.double() @ Bt.double().T)
        if C is not None:
            exact += beta * C.double()
        exact += gamma * torch.eye(M, N, dtype=torch.float64, device=dev)
        assert _rel(new, exact.cpu().numpy()) <= REL_TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _native.lib()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    M = N = K = 2048            # 4 (M + N) K = 32 MiB > 16 MiB
    assert 4 * (M + N) * K > SCRATCH_BYTES
    A = torch.zeros(M, K, device=dev)
    Bt = torch.zeros(N, K, device=dev)
    D = torch.full((M, N), 3.0, device=dev)
    rc = _call(lib.fx_product_f32_noalloc, M, N, K, A, Bt, 1.0, 0.0, None, 0.0, D, stream)
    assert rc == _native.ERR_VALUE
    assert b"scratch" in lib.fx_product_error()
    torch.cuda.synchronize()
    assert bool((D == 3.0).all())          # nothing was launched


def test_noalloc_rejects_sizes_whose_scratch_arithmetic_would_wrap():
    """Sizes far beyond the array are rejected before any arithmetic on them: with M = 2^60 the
    scratch size 4 (M + N) K wraps around 64 bits to a small number, which a check of the product
    alone would let through.  Nothing is launched, so the small operands are never read."""
    import torch
    lib = _native.lib()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    A = torch.zeros(16, 64, device=dev)
    Bt = torch.zeros(16, 64, device=dev)
    D = torch.full((16, 16), 3.0, device=dev)
    for M, N, K in [(1 << 60, 16, 64), (16, 1 << 60, 64), (16, 16, 1 << 40)]:
        assert (4 * (M + N) * K) % (1 << 64) < SCRATCH_BYTES or K > 32768
        rc = lib.fx_product_f32_noalloc(M, N, K, _p(A), 64, _p(Bt), 64, 1.0, 0.0, None, 0, 0.0,
                                        _p(D), 16, stream)
        assert rc == _native.ERR_VALUE, (M, N, K)
        assert b"at most" in lib.fx_product_error()
    torch.cuda.synchronize()
    assert bool((D == 3.0).all())
