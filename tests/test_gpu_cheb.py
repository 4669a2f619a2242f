"""The Chebyshev-Bessel approximant of walk generators (FX_OPT_APPROX = 1; needs a GPU).

In place of the Pade approximant and its solve, exp(iB / 2^s) is the Chebyshev series of
e^{iaz} in Z = B / rho (rho a spectral bound of B, a = rho / 2^s) truncated at the plan's
degree, evaluated with products of commuting real symmetric matrices only, then squared s
times.  Checked against the FP64 eigendecomposition at the parity bar (complex64 U within 1e-5
relative, states at infidelity <= 1e-10, including the state at the spectrum's two ends, which
a truncation error hits hardest), in both forms; the plan the device reports against
fx_chebyshev_plan at the device's own spectral bound and against the CPU statement of the plan.
"""
import math

import numpy as np
import pytest

from oracle import cheb_oracle as co
from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

C64_REL = 1e-5
INFID = 1e-10


def _laplacian_generator(A, t):
    L = np.diag(A.sum(axis=1)) - A
    return np.asarray(-1j * (-1.0 * L) * t, dtype=np.complex64)


def _eig(X):
    import torch
    lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to("cuda"))
    return lam, V


def _walk(X, form, approx, selector="plain"):
    import torch
    from fastctqw_b200._native import Engine
    n = X.shape[0]
    dev = torch.device("cuda", 0)
    dX = torch.from_numpy(X).to(dev)
    p0 = torch.zeros(n, dtype=torch.complex64, device=dev)
    p0[0] = 1.0
    dp = torch.empty_like(p0)
    dU = torch.empty_like(dX)
    e = Engine(n, np.complex64)
    e.configure(form=form, approx=approx, selector=selector)
    e.walk_device(dX, p0, dp, dU)
    torch.cuda.synchronize()
    out = (dU.cpu().numpy(), dp.cpu().numpy(), e.stats(), e.spectral_radius())
    e.close()
    return out


@pytest.mark.parametrize("n,form", [(1024, "plain"), (2048, "mixed"), (4096, "plain"), (4096, "mixed")])
def test_chebyshev_walk_meets_the_bar(n, form):
    import torch
    from fastctqw_b200 import _native, graphs
    A = graphs.erdos_renyi(n, 0.5, seed=11, dtype=np.float32)
    X = _laplacian_generator(A, 4.5)
    lam, V = _eig(X)
    Vc = V.to(torch.complex128)
    Uref = ((Vc * torch.exp(1j * lam)) @ Vc.T).cpu().numpy()
    U, psi, st, sp = _walk(X, form, "chebyshev")
    assert st["m"] == 0 and st["solver"] == 3 and st["sel_outcome"] == 5, st
    plan = _native.chebyshev_plan(sp["upper_bound"])
    assert (st["s"], st["degree"]) == (plan["s"], plan["degree"]), (st, plan)
    assert eo.rel_error(U, Uref) <= C64_REL, eo.rel_error(U, Uref)
    assert eo.infidelity(psi, Uref[:, 0]) <= INFID
    U128 = U.astype(np.complex128)
    for p0 in (graphs.uniform_state(n), graphs.random_state(n, 3)):
        p = p0.astype(np.complex128)
        assert eo.infidelity(U128 @ p, Uref @ p) <= INFID
    # the two ends of the spectrum, where a truncation error is largest
    Vn = V.cpu().numpy()
    p = (Vn[:, 0] + Vn[:, -1]) / math.sqrt(2.0)
    assert eo.infidelity(U128 @ p, Uref @ p) <= INFID


def test_estimated_selection_takes_the_lanczos_bound():
    """With the estimated selection the polynomial is planned on min(rigorous bound, 1.25 x the
    Lanczos estimate), which is the smaller one on dense graphs: fewer products, same bar."""
    import torch
    from fastctqw_b200 import _native, graphs
    n = 2048
    A = graphs.erdos_renyi(n, 0.5, seed=5, dtype=np.float32)
    X = _laplacian_generator(A, 4.5)
    lam, V = _eig(X)
    Vc = V.to(torch.complex128)
    Uref = ((Vc * torch.exp(1j * lam)) @ Vc.T).cpu().numpy()
    U, psi, st, sp = _walk(X, "plain", "chebyshev", selector="estimated")
    rho = min(sp["upper_bound"], 1.25 * sp["lanczos"])
    assert rho < sp["upper_bound"]
    # the spectrum of the shifted generator (trace shift mu, the all-ones mode, eigenvalue 0 of a
    # Laplacian, moved to 0 by the rank-one shift) lies inside [-rho, rho]
    lamn = lam.cpu().numpy()
    mu = float(np.trace(X.imag.astype(np.float64))) / n
    rho_true = float(np.max(np.abs(np.delete(lamn, np.argmin(np.abs(lamn))) - mu)))
    assert sp["lanczos"] <= rho_true * (1 + 1e-9) and rho_true <= rho
    # phase 1 computed A2 only: the cap is min(||Y||_1, ||A2||_1^(1/2)), still rigorous
    assert rho_true <= sp["upper_bound"]
    assert st["gemm_launches"] < _walk(X, "plain", "chebyshev", selector="plain")[2]["gemm_launches"]
    plan = _native.chebyshev_plan(rho)
    assert (st["s"], st["degree"]) == (plan["s"], plan["degree"]), (st, plan)
    assert eo.rel_error(U, Uref) <= C64_REL
    assert eo.infidelity(psi, Uref[:, 0]) <= INFID


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_chebyshev_batch_of_uneven_and_long_walks(form):
    """Uneven walks (random regular and G(n, p), adjacency and Laplacian, t up to 1000: up to ~15
    squarings) in one grouped batch, against the FP64 eigendecomposition on psi0 = (v_max +
    v_min) / sqrt 2; every walk reports the polynomial (m = 0, outcome 5)."""
    import torch
    from fastctqw_b200 import selector
    from fastctqw_b200.batch import WalkBatch
    dev = torch.device("cuda", 0)
    walks = [w for w, _ in zip(selector.make_walks(40, 17, 64, 1536, 0.1, 1000.0), range(40))]
    Xs = [X for X, _ in walks]
    dX = [torch.from_numpy(X).to(dev) for X in Xs]
    p0s, refs = [], []
    for X in Xs:
        lam, V = _eig(X)
        p0s.append(((V[:, -1] + V[:, 0]) / math.sqrt(2.0)).to(torch.complex64))
        refs.append((torch.exp(1j * lam[-1]) * V[:, -1] + torch.exp(1j * lam[0]) * V[:, 0]) / math.sqrt(2.0))
    outs = [torch.empty_like(p) for p in p0s]
    with WalkBatch([X.shape[0] for X in Xs], form=form, approx="chebyshev") as b:
        b.run_device(dX, p0s, outs)
        torch.cuda.synchronize()
        m, s = b.selection()
        det = b.details()
    assert (m == 0).all(), m
    assert (np.asarray(det["outcome"]) == 5).all(), det["outcome"]
    assert s.max() >= 10, s
    for k, (q, ref) in enumerate(zip(outs, refs)):
        q = q.to(torch.complex128)
        inf = float(1.0 - torch.vdot(ref, q).abs() ** 2 / (torch.vdot(q, q).real * torch.vdot(ref, ref).real))
        assert inf <= INFID, (form, walks[k][1], int(s[k]), inf)


def test_chebyshev_small_and_degenerate_walks():
    """Sizes 1, 2, 3, 17 and a zero generator (t = 0: degree 0, no squaring, U = I exactly), in
    one batch, against the FP64 propagator; the polynomial's plan at the device's spectral bound
    is the CPU statement's."""
    import torch
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import WalkBatch
    dev = torch.device("cuda", 0)
    gens = []
    for n, t in ((1, 2.0), (2, 0.7), (3, 40.0), (17, 3.0), (33, 0.0)):
        A = np.ones((n, n), dtype=np.float32) - np.eye(n, dtype=np.float32) if n < 17 else \
            graphs.erdos_renyi(n, 0.4, seed=n, dtype=np.float32)
        gens.append(np.asarray(-1j * (-1.0 * A) * t, dtype=np.complex64))
    with WalkBatch([X.shape[0] for X in gens], approx="chebyshev") as b:
        outs = b.run(gens, [graphs.uniform_state(X.shape[0]) for X in gens])
        m, s = b.selection()
        sp = b.spectral()
    for k, X in enumerate(gens):
        n = X.shape[0]
        lam, V = np.linalg.eigh(X.imag.astype(np.float64))
        ref = (V * np.exp(1j * lam)) @ (V.T @ graphs.uniform_state(n).astype(np.complex128))
        assert eo.infidelity(outs[k].astype(np.complex128), ref) <= INFID, (k, n)
        plan = co.plan(float(sp["upper_bound"][k]))
        assert int(s[k]) == plan["s"] and m[k] == 0, (k, s[k], plan)
    assert int(s[-1]) == 0 and np.allclose(outs[-1], graphs.uniform_state(33), atol=0, rtol=0)


def test_chebyshev_complex128_walk_plans_a_tighter_bound():
    """complex128 walks plan the polynomial at error 1e-12 (complex64 at 1e-6), so that the
    truncation stays far below the int8 products' own rounding: U as close to the FP64
    propagator as the Pade approximant's on the same walk (both bound by the 35-bit slices)."""
    import torch
    from fastctqw_b200 import _native, graphs
    from fastctqw_b200._native import Engine
    n = 600
    A = graphs.erdos_renyi(n, 0.3, seed=8, dtype=np.float64)
    L = np.diag(A.sum(axis=1)) - A
    X = np.asarray(-1j * (-1.0 * L) * 3.0, dtype=np.complex128)
    lam, V = np.linalg.eigh(X.imag)
    Uref = (V * np.exp(1j * lam)) @ V.T
    dev = torch.device("cuda", 0)
    dX = torch.from_numpy(X).to(dev)
    out = {}
    for approx in ("pade", "chebyshev"):
        dU = torch.empty_like(dX)
        e = Engine(n, np.complex128)
        e.configure(form="plain", approx=approx)
        e.run_device(dX, dU)
        torch.cuda.synchronize()
        out[approx] = (e.stats(), e.spectral_radius(), eo.rel_error(dU.cpu().numpy(), Uref))
        e.close()
    st, sp, err = out["chebyshev"]
    plan = _native.chebyshev_plan(sp["upper_bound"], 1e-12)
    assert st["m"] == 0 and (st["s"], st["degree"]) == (plan["s"], plan["degree"]), (st, plan)
    assert plan["cost"] >= _native.chebyshev_plan(sp["upper_bound"])["cost"]
    print(f"complex128 N = {n}: U within {err:.2e} (Chebyshev) and {out['pade'][2]:.2e} (Pade) of FP64")
    assert err <= 1e-7 and err <= 1.5 * out["pade"][2]
