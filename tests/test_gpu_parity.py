"""Parity of the B200 engine with the oracle and the reference's fixtures (needs a GPU).

Tolerances (stated per test): complex64 handles must match U within 1e-5 relative
(Frobenius) of the FP64 result; walk states must reach infidelity <= 1e-10 against the FP64
eigendecomposition propagator; complex128 handles within 1e-10 relative.
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

C64_REL = 1e-5
C128_REL = 1e-10
INFID = 1e-10


@pytest.fixture(scope="module")
def fe():
    from fastctqw_b200 import fastexpm
    return fastexpm


def _run(fe, X, form=None, **kw):
    cls = {np.dtype(np.complex64): fe.ExpMatComplex64, np.dtype(np.complex128): fe.ExpMatComplex128,
           np.dtype(np.float32): fe.ExpMatFloat32, np.dtype(np.float64): fe.ExpMatFloat64}[X.dtype]
    with cls(X.shape[0]) as e:
        if form or kw:
            e.configure(**({"form": form} if form else {}), **kw)
        U = e.run(X)
        st = e.stats()
    return U, st


def test_native_library_is_loaded():
    from fastctqw_b200 import _native
    assert _native.device_ok()
    assert b"sm_100a" in _native.lib().fx_version()


@pytest.mark.parametrize("form", ["plain", "simt"])
def test_reference_expm_fixtures_c64(golden, fe, form):
    for name, c in golden.items():
        if "X" not in c or c["X"].dtype != np.complex64:
            continue
        U, st = _run(fe, c["X"], form)
        ref = c["U_scipy_f64"]
        assert eo.rel_error(U, ref) < C64_REL, (name, eo.rel_error(U, ref), st)


def test_reference_expm_fixtures_c128(golden, fe):
    for name, c in golden.items():
        if "X" not in c or c["X"].dtype != np.complex128:
            continue
        U, st = _run(fe, c["X"])
        assert eo.rel_error(U, c["U_scipy"]) < C128_REL, (name, eo.rel_error(U, c["U_scipy"]), st)


def test_reference_walk_fixtures(golden):
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    for name, c in golden.items():
        if "psi_ref_e0" not in c:
            continue
        A = c["A"]
        # The oracle runs on the same (rounded) input X as the engine: for complex64 data the
        # rounding of X itself moves expm(X) away from the FP64 truth of the exact H by up to
        # ||dX||_2 (about 1e-5 for the t = 100 weighted case, where even the exact expm of the
        # rounded X has infidelity 4.3e-10 against the exact H), which is not an error of the
        # engine.  Against the exact H the engine must do no worse than the reference's own
        # result (psi_ref, scipy.linalg.expm in the input precision).
        dt = np.complex64 if A.dtype == np.float32 else np.complex128
        H = eo.build_hamiltonian(A, float(c["gamma"]), bool(c["laplacian"]), dtype=dt)
        Uo = eo.expm(eo.walk_generator(H, float(c["t"]), dt).astype(np.complex128))
        for kind in ("uniform", "e0", "random"):
            w = Ctqw(A, State(c[f"psi0_{kind}"]), float(c["gamma"]), bool(c["laplacian"]))
            w.runWalk(float(c["t"]))
            psi = w.getFinalState().getState()
            inf = eo.infidelity(psi, Uo @ c[f"psi0_{kind}"].astype(np.complex128))
            assert inf <= INFID, (name, kind, inf)
            inf_truth = eo.infidelity(psi, c[f"psi_eig_{kind}"])
            inf_ref = eo.infidelity(c[f"psi_ref_{kind}"], c[f"psi_eig_{kind}"])
            assert inf_truth <= max(INFID, inf_ref), (name, kind, inf_truth, inf_ref)
            if "U_eig" in c:
                U = w.getOperator().getOperator()
                tol = C64_REL if A.dtype == np.float32 else C128_REL
                assert eo.rel_error(U, Uo) < tol, (name, eo.rel_error(U, Uo))
            w.free()


def test_operator_build_matches_reference_output(golden):
    from fastctqw_b200.Operator import Operator
    for name, c in golden.items():
        if "U_ref" not in c:
            continue
        op = Operator(c["A"], float(c["gamma"]), bool(c["laplacian"]))
        op.buildExpmOperator(float(c["t"]))
        U = op.getOperator()
        assert U.dtype == c["U_ref"].dtype
        tol = 1e-4 if U.dtype == np.complex64 else 1e-9   # the reference's own c64 error
        assert eo.rel_error(U, c["U_ref"]) < tol, name
        op.free()


def test_general_complex_sizes(N, fe):
    """Arbitrary complex input (the reference's perf-test family, A_real + 1j*rand)."""
    rng = np.random.default_rng(N)
    for scale in (0.05, 1.0, 8.0):
        X = (scale * (rng.standard_normal((N, N)) + 1j * rng.random((N, N))) / max(1.0, np.sqrt(N)))
        ref = eo.expm(X)
        for dt, tol in ((np.complex64, C64_REL), (np.complex128, C128_REL)):
            U, st = _run(fe, X.astype(dt))
            assert eo.rel_error(U, ref) < tol * max(1.0, np.linalg.cond(ref) / 10), (N, scale, dt, st)


def test_selection_matches_oracle(fe):
    rng = np.random.default_rng(4)
    for n in (16, 64, 200):
        for scale in (1e-3, 0.1, 1.0, 5.0, 60.0):
            X = scale * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
            _, sel = eo.expm(X, shift="auto", structure=True, return_selection=True)
            _, st = _run(fe, X.astype(np.complex128))
            assert (st["m"], st["s"]) == (sel.m, sel.s), (n, scale, st, sel)


def test_structured_walk_selection_and_accuracy(fe):
    from fastctqw_b200 import graphs
    for n, t in ((256, 4.5), (512, 4.5)):
        A = graphs.erdos_renyi(n, 0.5, seed=n)
        H = eo.build_hamiltonian(A.astype(np.float64), 1.0, True)
        X = eo.walk_generator(H, t, np.complex64)
        _, sel = eo.expm(X.astype(np.complex128), shift="auto", structure=True, return_selection=True)
        U, st = _run(fe, X)
        assert st["structured"] == 1 and st["rank1_shift"] == 1
        assert (st["m"], st["s"]) == (sel.m, sel.s)
        Ue = eo.propagator_eigh(H, t)
        assert eo.rel_error(U, Ue) < C64_REL
        e0 = np.zeros(n)
        e0[0] = 1
        assert eo.infidelity(U @ e0, Ue @ e0) < INFID


def test_forms_agree(fe):
    from fastctqw_b200 import graphs
    A = graphs.erdos_renyi(300, 0.3, seed=1)
    H = eo.build_hamiltonian(A.astype(np.float64), 1.0, True)
    X = eo.walk_generator(H, 2.0, np.complex64)
    Ue = eo.propagator_eigh(H, 2.0)
    Up, _ = _run(fe, X, "plain")
    Us, _ = _run(fe, X, "simt")
    Um, _ = _run(fe, X, "mixed")
    assert eo.rel_error(Up, Ue) < C64_REL
    assert eo.rel_error(Us, Ue) < C64_REL
    assert eo.rel_error(Um, Ue) < 1e-2   # BF16 hi+lo (16 significant bits)


def test_real_handles(fe):
    rng = np.random.default_rng(2)
    A = rng.standard_normal((50, 50)) / 7
    ref = eo.expm(A)
    U32, _ = _run(fe, A.astype(np.float32))
    U64, _ = _run(fe, A.astype(np.float64))
    assert U32.dtype == np.float32 and U64.dtype == np.float64
    assert eo.rel_error(U32, ref) < C64_REL
    assert eo.rel_error(U64, ref) < C128_REL


def test_drop_in_errors(fe):
    with fe.ExpMatComplex64(4) as e:
        with pytest.raises(TypeError):
            e.run([[0.0] * 4] * 4)
        with pytest.raises(ValueError):
            e.run(np.zeros((3, 3), np.complex64))
        with pytest.raises(ValueError):
            e.run(np.full((4, 4), np.nan, np.complex64))


def test_forcecast_like_pybind(fe):
    X = (0.3j * np.ones((8, 8))).astype(np.complex128)
    with fe.ExpMatComplex64(8) as e:
        U = e.run(X)
    assert U.dtype == np.complex64
    assert eo.rel_error(U, eo.expm(X)) < C64_REL


def test_torch_device_handoff(fe):
    import torch
    n = 96
    rng = np.random.default_rng(3)
    X = (0.2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))).astype(np.complex64)
    dX = torch.from_numpy(X).cuda()
    dU = torch.empty_like(dX)
    with fe.ExpMatComplex64(n) as e:
        e.run_device(dX, dU)
        torch.cuda.synchronize()
    assert eo.rel_error(dU.cpu().numpy(), eo.expm(X)) < C64_REL


def test_repeatable_bitwise(fe):
    rng = np.random.default_rng(8)
    X = (rng.standard_normal((200, 200)) * 1j).astype(np.complex64)
    X = (X + X.T) / 2
    with fe.ExpMatComplex64(200) as e:
        U1 = e.run(X)
        U2 = e.run(X)
    assert np.array_equal(U1, U2)
