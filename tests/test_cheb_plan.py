"""The Chebyshev approximant's plan and arithmetic on the CPU (no GPU needed).

The device plans the polynomial stage on the host (fx_chebyshev_plan): the number of squarings
s, the degree D of the Chebyshev series of e^{iaz} in Z = B / rho and the baby steps m.  Checked
here one to one against the CPU statement of the plan (oracle/cheb_oracle.py), whose pieces are
checked in turn: its Bessel values against scipy, its truncation bound against the series'
actual error, the coefficient split and block decomposition against a direct evaluation of the
series, and the whole FP64 sequence of steps against the eigendecomposition propagator.
"""
import math

import numpy as np
import pytest
from scipy.special import jv

from oracle import cheb_oracle as co
from oracle import expm_oracle as eo


def _native_or_skip():
    from fastctqw_b200 import _native
    try:
        _native.lib()
    except ImportError as e:   # the library is built by __graft_entry__.build()
        pytest.skip(str(e))
    return _native


@pytest.mark.parametrize("a", [0.0, 1e-6, 0.3, 2.5, 8.9, 40.0, 300.0])
def test_bessel_values_match_scipy(a):
    j = co.bessel_j(a, 120)
    ref = jv(np.arange(121), a)
    assert np.max(np.abs(j - ref)) <= 1e-14 * max(1.0, a ** 0.5)


@pytest.mark.parametrize("a,tol", [(0.5, 1e-12), (8.9, 7.8e-9), (40.0, 1e-9), (250.0, 1e-8)])
def test_degree_bounds_the_series_error(a, tol):
    """The truncated series meets the bound on [-1, 1], and one degree less does not bound it."""
    D = co.degree(a, tol)
    z = np.cos(np.linspace(0.0, np.pi, 2001))
    J = co.bessel_j(a, D)
    k = np.arange(D + 1)
    coef = np.where(k == 0, 1.0, 2.0) * (1j ** k) * J
    series = np.polynomial.chebyshev.chebval(z, coef)
    assert np.max(np.abs(series - np.exp(1j * a * z))) <= tol
    if D > 0:
        J2 = co.bessel_j(a, D + 60)
        assert 2.0 * np.abs(J2[D:]).sum() > tol


@pytest.mark.parametrize("D,m", [(2, 2), (5, 1), (9, 2), (25, 3), (31, 3), (40, 2), (38, 5), (44, 4)])
def test_split_and_blocks_reproduce_the_series(D, m):
    """Even part in C = T_2(z), odd part z x (series in C), each summed over T_g(T_m(C)) blocks by
    Clenshaw's recurrence: the same values as the series itself."""
    a = 0.9 * D
    z = np.cos(np.linspace(0.0, np.pi, 301))
    J = co.bessel_j(a, D)
    k = np.arange(D + 1)
    coef = np.where(k == 0, 1.0, 2.0) * (1j ** k) * J
    direct = np.polynomial.chebyshev.chebval(z, coef)
    e, b = co.split_coefficients(a, D)
    C = 2.0 * z * z - 1.0

    def clen(x):
        r = co.blocks(x, m)
        T = [np.polynomial.chebyshev.chebval(C, [0.0] * k + [1.0]) for k in range(m + 1)]
        G = np.polynomial.chebyshev.chebval(C, [0.0] * m + [1.0])
        L = r.shape[0] - 1

        def rg(g):
            return sum(r[g, j] * T[j] for j in range(m))
        if L == 0:
            return rg(0)
        b1, b2 = rg(L), np.zeros_like(C)
        for g in range(L - 1, 0, -1):
            b1, b2 = 2.0 * G * b1 - b2 + rg(g), b1
        return G * b1 - b2 + rg(0)

    got = clen(e) + 1j * z * (clen(b) if len(b) else 0.0)
    assert np.max(np.abs(got - direct)) <= 1e-12


def test_plan_matches_the_cpu_statement():
    _native = _native_or_skip()
    rng = np.random.default_rng(0)
    rhos = [0.0, 1e-9, 1e-3, 0.1, 0.5, 1.0, 2.0, 8.0, 10.0, 100.0, 1294.0, 1755.0, 1e4, 1e6]
    rhos += list(10.0 ** rng.uniform(-4, 6, 60))
    for rho in rhos:
        a = _native.chebyshev_plan(rho)
        b = co.plan(rho)
        assert (a["s"], a["degree"], a["baby"], a["cost"]) == (b["s"], b["degree"], b["baby"], b["cost"]), rho
    with pytest.raises(ValueError):
        _native.chebyshev_plan(-1.0)
    with pytest.raises(ValueError):
        _native.chebyshev_plan(float("nan"))
    with pytest.raises(ValueError):
        _native.chebyshev_plan(1.0, 0.0)
    with pytest.raises(ValueError):   # no s <= 60 brings a = rho / 2^s below 1024
        _native.chebyshev_plan(1e25)
    assert _native.chebyshev_plan(1e20)["s"] >= 50


def test_plan_is_cheaper_than_pade_on_the_dense_walk():
    """N = 10000 dense Laplacian at t = 4.5: the rigorous bound 1755 and the Lanczos bound
    1.25 x 1035 take 31 and 29 products (6 squarings); the Pade stage with its Newton-Schulz solve
    and 7 squarings took 44."""
    assert co.plan(1755.0)["cost"] == 31
    p = co.plan(1.25 * 1035.0)
    assert (p["cost"], p["s"], p["baby"]) == (29, 6, 5)


@pytest.mark.parametrize("n,p,t", [(120, 0.5, 4.5), (90, 0.1, 60.0), (64, 0.3, 0.01)])
def test_fp64_steps_match_the_eigendecomposition(n, p, t):
    rng = np.random.default_rng(n)
    A = np.triu((rng.random((n, n)) < p).astype(np.float64), 1)
    A = A + A.T
    H = eo.build_hamiltonian(A, 1.0, True)
    B = -(H * t)
    lam, V = np.linalg.eigh(B)
    rho = np.abs(B).sum(axis=0).max()
    R, plan = co.walk_propagator(B, rho)
    Uref = (V * np.exp(1j * lam)) @ V.T
    assert eo.rel_error(R, Uref) <= 1e-6
    assert plan["s"] >= 0 and plan["degree"] >= 1
