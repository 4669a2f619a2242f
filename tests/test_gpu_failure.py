"""The failure path of the tensor-core product kernel (needs a GPU; faults nothing).

Every wait inside the product kernel (on an mbarrier of its TMA / MMA / epilogue roles) is
bounded by a deadline; when one runs out the kernel sets the device error word, drains what it
issued, frees its tensor memory and returns, and the host raises FX_ERR_TIMEOUT.  Here the
diagnostic option FX_OPT_INJECT_STALL makes one product launch leave the operand loads of one
K step out -- a dependency that nothing will ever satisfy -- with a 10 ms deadline: the run
must fail with the timeout status, and the next run on the same handle must succeed and be
correct.  No trap, no bad address, no unbounded wait.
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("launch", [0, 4])   # 0: a phase-1 power; 4: a Pade product of phase 2
def test_bounded_wait_runs_out_and_the_handle_recovers(launch):
    import torch
    from fastctqw_b200 import graphs
    from fastctqw_b200._native import Engine
    n, t = 256, 2.0
    A = graphs.random_regular(n, 5, seed=31)
    X = np.asarray(1j * A * np.float32(t), dtype=np.complex64)        # X = -1j H t, H = -A
    p0 = graphs.random_state(n, 5)
    dev = torch.device("cuda", 0)
    dX = torch.from_numpy(X).to(dev)
    dp0 = torch.from_numpy(p0).to(dev)
    dp = torch.empty_like(dp0)
    e = Engine(n, np.complex64)
    e.walk_device(dX, dp0, dp)                 # a good run first (records the launch graphs)
    torch.cuda.synchronize()
    e.configure(timeout_ms=10, inject_stall=launch)
    with pytest.raises(RuntimeError, match="timed out"):
        e.walk_device(dX, dp0, dp)
        torch.cuda.synchronize()
    e.configure(timeout_ms=2000, inject_stall=-1)
    dp.fill_(float("nan"))
    e.walk_device(dX, dp0, dp)
    torch.cuda.synchronize()
    lam, V = np.linalg.eigh(A.astype(np.float64))
    ref = (V * np.exp(1j * lam * float(np.float32(t)))) @ (V.T @ p0.astype(np.complex128))
    assert eo.infidelity(dp.cpu().numpy(), ref) <= 1e-10
    e.close()


@pytest.mark.parametrize("k", [0, 1, 5])
def test_injected_allocation_failure_is_a_memory_error(k, monkeypatch):
    """FX_INJECT_ALLOC_FAIL=k makes the k-th workspace allocation fail as if the device were
    full: the call raises MemoryError (FX_ERR_NOMEM), nothing is left half-built, and the same
    handle (and a new batch) work once the variable is gone.  Host-side only: no GPU fault."""
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import WalkBatch
    from fastctqw_b200.fastexpm import ExpMatComplex64
    n, t = 200, 1.5
    A = graphs.random_regular(n, 4, seed=3)
    X = np.asarray(1j * A * np.float32(t), dtype=np.complex64)
    ref = eo.propagator_eigh(-A.astype(np.float64), t)
    e = ExpMatComplex64(n)
    monkeypatch.setenv("FX_INJECT_ALLOC_FAIL", str(k))
    with pytest.raises(MemoryError):
        e.run(X)
        for _ in range(8):   # later allocations of the first runs, until the k-th
            e.run(X)
    monkeypatch.delenv("FX_INJECT_ALLOC_FAIL")
    assert eo.rel_error(e.run(X), ref) <= 1e-5
    e.free()
    monkeypatch.setenv("FX_INJECT_ALLOC_FAIL", str(k))
    with pytest.raises(MemoryError):
        b = WalkBatch([n, n // 2])
        b.run([X, X[: n // 2, : n // 2]])
    monkeypatch.delenv("FX_INJECT_ALLOC_FAIL")
    with WalkBatch([n]) as b:
        psi = b.run([X], [graphs.uniform_state(n)])[0]
    assert eo.infidelity(psi.astype(np.complex128), ref @ graphs.uniform_state(n).astype(np.complex128)) <= 1e-10
