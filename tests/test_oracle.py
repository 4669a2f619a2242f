"""Pin the CPU oracle before trusting it (CPU only).

* golden fixtures generated from the reference's own CPU path (tests/golden/make_golden.py),
* the FP64 eigendecomposition propagator,
* scipy's own known-answer tests for expm, run with the oracle substituted.
"""
import importlib
import math

import numpy as np
import pytest
import scipy.linalg as sl

from oracle import expm_oracle as eo


def test_pade_coefficients_match_published_tables():
    # Higham (2005) Table 2.2 values, as printed in scipy/sparse/linalg/_matfuncs.py:489-526.
    assert eo.pade_coefficients(3) == [120., 60., 12., 1.]
    assert eo.pade_coefficients(5) == [30240., 15120., 3360., 420., 30., 1.]
    assert eo.pade_coefficients(7)[0] == 17297280. and eo.pade_coefficients(7)[-2] == 56.
    assert eo.pade_coefficients(9)[0] == 17643225600.
    assert eo.pade_coefficients(13)[0] == 64764752532480000.
    assert eo.pade_coefficients(13)[-2] == 182.


def test_ell_constants():
    assert eo.ell_constant(3) == 100800.
    assert eo.ell_constant(5) == 10059033600.
    assert eo.ell_constant(7) == 4487938430976000.
    assert math.isclose(eo.ell_constant(13), 1.1325077560602111e35, rel_tol=1e-15)


@pytest.mark.parametrize("shift", ["none", "trace", "auto"])
def test_oracle_vs_reference_walk_fixtures(golden, shift):
    for name, c in golden.items():
        if "U_ref" not in c:
            continue
        A = c["A"]
        H = eo.build_hamiltonian(A, float(c["gamma"]), bool(c["laplacian"]))
        X = eo.walk_generator(H, float(c["t"]))
        U = eo.expm(X, shift=shift, structure=True)
        # The reference ran in its input precision; the eigh propagator is the FP64 truth.
        assert eo.rel_error(U, c["U_eig"]) < 1e-10, name
        tol = 1e-4 if c["U_ref"].dtype == np.complex64 else 1e-10
        assert eo.rel_error(U, c["U_ref"]) < tol, name


def test_oracle_vs_reference_expm_fixtures(golden):
    for name, c in golden.items():
        if "X" not in c:
            continue
        X = c["X"].astype(np.complex128)
        U = eo.expm(X)
        ref = c.get("U_scipy_f64", c["U_scipy"])
        assert eo.rel_error(U, ref) < 1e-11, name
        if "U_taylor" in c:
            assert eo.rel_error(U, c["U_taylor"]) < 1e-9, name


def test_oracle_walk_states(golden):
    for name, c in golden.items():
        if "psi_ref_e0" not in c:
            continue
        H = eo.build_hamiltonian(c["A"], float(c["gamma"]), bool(c["laplacian"]))
        X = eo.walk_generator(H, float(c["t"]))
        U = eo.expm(X, shift="auto", structure=True)
        for kind in ("uniform", "e0", "random"):
            psi = U @ c[f"psi0_{kind}"].astype(np.complex128)
            assert eo.infidelity(psi, c[f"psi_eig_{kind}"]) < 1e-20 + 1e-12, (name, kind)
            # The reference itself (complex64 path) is within its own precision.
            tol = 1e-6 if c["A"].dtype == np.float32 else 1e-12
            assert eo.infidelity(c[f"psi_ref_{kind}"], c[f"psi_eig_{kind}"]) < tol, (name, kind)


def test_shift_identities():
    rng = np.random.default_rng(5)
    n = 40
    # Every row/column sum equal -> rank-one shift applies.
    a = (rng.random((n, n)) < 0.3).astype(float)
    a = np.triu(a, 1)
    a = a + a.T
    L = np.diag(a.sum(1)) - a
    # 0.8 is not a binary fraction: the rounded entries leave row sums of order 1e-16 instead
    # of exact zeros.  The shift still applies (the line sums agree to rounding level) and the
    # result stays exact to rounding.
    X8 = 1j * 0.8 * L
    assert eo.preprocess(X8, "auto")[1].rank1
    assert eo.rel_error(eo.expm(X8, shift="auto", structure=True), sl.expm(X8)) < 1e-12
    # Row sums that differ by more than rounding: no rank-one shift.
    b = np.ones((n, n)) - np.eye(n)
    b[0, 1] = b[1, 0] = 1.0 + 1e-9
    assert not eo.preprocess(1j * b, "auto")[1].rank1
    assert eo.preprocess(1j * (np.ones((n, n)) - np.eye(n)), "auto")[1].rank1
    X = 1j * 0.75 * L
    Y, sh = eo.preprocess(X, "auto")
    assert sh.rank1
    assert np.allclose(Y.sum(axis=1), 0, atol=1e-12)
    U = eo.expm(X, shift="auto", structure=True)
    assert eo.rel_error(U, sl.expm(X)) < 1e-12
    # General complex: only the trace shift.
    G = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    Y, sh = eo.preprocess(G, "auto")
    assert not sh.rank1
    assert eo.rel_error(eo.expm(G, shift="auto"), sl.expm(G)) < 1e-12


def test_structured_selection_never_larger():
    """Dropping l for skew-Hermitian inputs can only lower s, and stays accurate."""
    rng = np.random.default_rng(9)
    for n, t in ((60, 4.5), (90, 30.0)):
        a = (rng.random((n, n)) < 0.5).astype(float)
        a = np.triu(a, 1)
        a = a + a.T
        H = eo.build_hamiltonian(a, 1.0, True)
        X = eo.walk_generator(H, t)
        U0, s0 = eo.expm(X, shift="auto", structure=False, return_selection=True)
        U1, s1 = eo.expm(X, shift="auto", structure=True, return_selection=True)
        assert s1.s <= s0.s
        assert eo.rel_error(U1, eo.propagator_eigh(H, t)) < 1e-11


def test_selection_matches_scipy_exact_norm_path(monkeypatch):
    """(m, s) agree with scipy.sparse.linalg._expm(use_exact_onenorm=True) on seeded cases."""
    mf = importlib.import_module("scipy.sparse.linalg._matfuncs")
    seen = {}
    orig = {m: getattr(mf._ExpmPadeHelper, f"pade{m}") for m in (3, 5, 7, 9)}
    orig13 = mf._ExpmPadeHelper.pade13_scaled

    def mk(m):
        def f(self):
            seen["ms"] = (m, 0)
            return orig[m](self)
        return f

    for m in (3, 5, 7, 9):
        monkeypatch.setattr(mf._ExpmPadeHelper, f"pade{m}", mk(m))

    def p13(self, s):
        seen["ms"] = (13, s)
        return orig13(self, s)

    monkeypatch.setattr(mf._ExpmPadeHelper, "pade13_scaled", p13)
    rng = np.random.default_rng(1)
    agree = 0
    total = 0
    for scale in (1e-3, 1e-2, 0.1, 0.5, 1.0, 3.0, 10.0, 100.0):
        for n in (5, 20):
            A = scale * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(n)
            mf._expm(A, use_exact_onenorm=True)
            _, sel = eo.expm(A, return_selection=True)
            total += 1
            agree += seen["ms"] == (sel.m, sel.s)
    # The d8/d10 estimates are lower bounds of the exact norms scipy uses here; they agree
    # on (nearly) every seeded case.
    assert agree >= total - 1, (agree, total)


SCIPY_KAT = ["test_zero_ndarray", "test_padecases_dtype_float", "test_padecases_dtype_complex",
             "test_logm_consistency", "test_integer_matrix", "test_integer_matrix_2",
             "test_pascal"] + [f"test_burkardt_{i}" for i in range(1, 15)]


@pytest.mark.parametrize("name", SCIPY_KAT)
def test_scipy_known_answers_with_oracle(name, monkeypatch):
    """scipy's TestExpM known-answer cases (scipy/sparse/linalg/tests/test_matfuncs.py),
    imported from the installed scipy and run with the oracle in place of its expm."""
    tm = importlib.import_module("scipy.sparse.linalg.tests.test_matfuncs")

    import scipy.sparse as sp

    def oracle_expm(A):
        if sp.issparse(A):
            return sp.csc_array(oracle_expm(A.toarray()))
        A = np.asarray(A)
        if A.dtype.kind in "iub":
            A = A.astype(float)
        out = eo.expm(A)
        if A.dtype == np.float32:
            return out.astype(np.float32)
        if A.dtype == np.complex64:
            return out.astype(np.complex64)
        return out

    monkeypatch.setattr(tm, "expm", oracle_expm)
    getattr(tm.TestExpM(), name)()
