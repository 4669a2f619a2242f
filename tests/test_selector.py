"""Learned (m, s) selector, CPU parts: the network oracle and the certified truncation bound."""
import math

import numpy as np

from oracle import mlp_oracle as mo
from oracle import expm_oracle as eo


def test_oracle_gradient_matches_finite_differences():
    from fastctqw_b200 import selector
    rng = np.random.default_rng(0)
    w = selector.init_weights(3).astype(np.float64) + 0.01 * rng.standard_normal(5126)
    x = rng.standard_normal((17, 8))
    ym = rng.integers(0, 5, 17)
    ys = rng.random(17) * 10
    loss, g = mo.loss_grad(w, x, ym, ys, 0.3)
    for i in rng.choice(5126, 40, replace=False):
        e = np.zeros(5126)
        e[i] = 1e-6
        fd = (mo.loss_grad(w + e, x, ym, ys, 0.3)[0] - mo.loss_grad(w - e, x, ym, ys, 0.3)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_phase_error_is_the_pade_error_on_the_imaginary_axis():
    from fastctqw_b200 import selector
    for m in selector.DEGREES:
        b = eo.pade_coefficients(m)
        for x in (0.3, 1.7, 4.0):
            z = 1j * x
            p = sum(b[j] * z ** j for j in range(m + 1))
            q = sum(b[j] * (-z) ** j for j in range(m + 1))
            r = p / q
            assert abs(abs(r) - 1.0) < 1e-14
            assert abs(np.angle(r * np.exp(-1j * x)) - selector.phase_error(m, x)) < 1e-12


def test_certified_choice_bounds_the_exact_error_and_beats_double_precision_scaling():
    """The certified (m, s) keeps the exact phase error of every eigenvalue within tolerance,
    and needs fewer squarings than the double-precision selection for walk generators."""
    from fastctqw_b200 import graphs, selector
    rng = np.random.default_rng(2)
    saved = 0
    for k in range(6):
        n = int(rng.integers(60, 200))
        A = graphs.erdos_renyi(n, 0.3, seed=k, dtype=np.float64)
        t = float(rng.uniform(1, 40))
        X = -1j * (-A) * t
        Y, sh = eo.preprocess(X, "auto")
        B = (Y / 1j).real
        lam = np.linalg.eigvalsh(B)
        A2 = Y @ Y
        A4 = A2 @ A2
        A6 = A4 @ A2
        rho_up = min(eo.onenorm(Y), eo.onenorm(A4) ** 0.25, eo.onenorm(A6) ** (1 / 6))
        assert rho_up >= np.abs(lam).max() * (1 - 1e-12)
        m, s = selector.certified_choice(rho_up)
        err = np.max(np.abs(2.0 ** s * selector.phase_error(m, lam / 2.0 ** s)))
        assert err <= selector.PHASE_TOL
        plain = eo.select_pade(Y, normal=True)
        assert selector.PRODUCTS[m] + s <= selector.PRODUCTS[plain.m] + plain.s
        saved += selector.PRODUCTS[plain.m] + plain.s - selector.PRODUCTS[m] - s
    assert saved >= 6


def test_weight_folding_is_exact():
    from fastctqw_b200 import selector
    rng = np.random.default_rng(5)
    w = selector.init_weights(1).astype(np.float64)
    mean, std = rng.standard_normal(8), rng.random(8) + 0.5
    x = rng.standard_normal((9, 8))
    a = mo.forward(w, (x - mean) / std)[0]
    b = mo.forward(selector.fold_standardisation(w, mean, std), x)[0]
    assert np.allclose(a, b, atol=1e-10)
