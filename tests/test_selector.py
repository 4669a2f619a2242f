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


def test_lanczos_radius_is_a_sharp_lower_estimate():
    """The Lanczos estimate behind the estimated selection never exceeds the spectral radius and
    is within a few percent of it on the dense Laplacian family, while the rigorous norm bound
    sits about 1.5x above; the tridiagonal step agrees with a dense eigensolver."""
    from fastctqw_b200 import graphs
    n = 512
    A = graphs.erdos_renyi(n, 0.5, seed=3, dtype=np.float64)
    B = 4.5 * (np.diag(A.sum(1)) - A)
    Y = B - np.trace(B) / n * np.eye(n)
    Y -= Y.sum() / n * np.ones((n, n)) / n
    rho = np.abs(np.linalg.eigvalsh(Y)).max()
    est = eo.lanczos_radius(Y, steps=30)
    assert est <= rho * (1 + 1e-10) and est >= 0.95 * rho, (est, rho)
    A4 = np.linalg.matrix_power(Y, 4)
    bound = min(eo.onenorm(Y), eo.onenorm(A4) ** 0.25)
    assert bound >= 1.3 * rho
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(12), np.abs(rng.standard_normal(11)) + 0.1
    T = np.diag(a) + np.diag(b, 1) + np.diag(b, -1)
    assert abs(eo.tridiag_radius(a, b) - np.abs(np.linalg.eigvalsh(T)).max()) <= 1e-12 * np.abs(a).max()


def test_learned_gate_and_estimated_rule_use_the_lanczos_radius():
    """The Python mirror of the engine's selection: the gate of a learned proposal tests the
    phase bound at min(rho_up, 1.1 rho_L) with tolerance 1e-5; the estimated rule takes the
    cheapest choice that bound certifies at 1e-6."""
    from fastctqw_b200 import selector
    f = np.zeros((1, 8), dtype=np.float64)
    f[0, 1] = f[0, 6] = f[0, 7] = np.log2(3000.0)   # rho_up = 3000
    f[0, 4] = np.log2(800.0)                         # rho_L = 800 -> 880 with the margin
    m, s = selector.estimated_choice(f)
    assert (m[0], s[0]) == selector.certified_choice(880.0)
    mr, sr = selector.certified_choice(3000.0)
    assert selector.PRODUCTS[int(m[0])] + s[0] < selector.PRODUCTS[mr] + sr
    # a proposal at the gate's own tolerance is cheaper than the estimated choice: accepted
    pm, ps = selector.certified_choice(880.0, selector.GATE_TOL)
    assert selector.PRODUCTS[pm] + ps < selector.PRODUCTS[int(m[0])] + s[0]
    out = selector.gate(f, np.array([13]), np.array([12]), np.array([pm]), np.array([ps]))
    assert out[0] == 2
    # one squaring fewer fails the gate: the estimated choice is used
    out = selector.gate(f, np.array([13]), np.array([12]), np.array([pm]), np.array([ps - 1]))
    assert out[0] == 3
    # with a plain choice cheaper than the estimated one, a rejected proposal keeps the plain one
    cp = selector.PRODUCTS[int(m[0])] + s[0] - 1
    out = selector.gate(f, np.array([13]), np.array([cp - 6]), np.array([pm]), np.array([ps - 1]))
    assert out[0] == (-1 if selector.PRODUCTS[pm] + ps - 1 < cp else 0)


def test_label_sweep_resumes_from_its_chunk_cache(tmp_path):
    """A measured sweep keeps every finished chunk on disk, keyed by the sweep's arguments, and
    reads back the chunks it finds: here every chunk is already there, so the sweep returns them
    without touching a GPU, in order, with the walks' descriptions."""
    from fastctqw_b200 import selector
    args = dict(count=5, seed=11, nmin=64, nmax=96, tmin=0.1, tmax=1000.0, chunk=2, depth=5, form="plain")
    walks = [mt for _, mt in selector.make_walks(5, 11, 64, 96, 0.1, 1000.0)]
    sizes = (2, 2, 1)
    start = 0
    for index, k in enumerate(sizes):
        arr = {key: np.arange(start, start + k, dtype=np.float64) for key in selector.CHUNK_KEYS}
        arr["features"] = np.full((k, 8), float(index), dtype=np.float32)
        path = selector.chunk_cache_path(str(tmp_path), index, **args)
        selector.save_chunk(path, arr, walks[start:start + k])
        start += k
    other = selector.chunk_cache_path(str(tmp_path), 0, **dict(args, seed=12))
    assert other != selector.chunk_cache_path(str(tmp_path), 0, **args)
    ds = selector.make_dataset_measured(cache_dir=str(tmp_path), **args)
    assert np.array_equal(ds["label_m"], np.arange(5))
    assert ds["features"].shape == (5, 8) and list(ds["features"][:, 0]) == [0, 0, 1, 1, 2]
    assert [tuple(m) for m in ds["meta"]] == walks
    assert not any(p.name.endswith(".part.npz") for p in tmp_path.iterdir())
