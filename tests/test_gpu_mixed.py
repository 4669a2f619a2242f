"""The mixed (reduced-precision) form of the walk-generator pipeline (needs a GPU).

For walks padded to 4096 or more the mixed form slices the powers, the Pade and solve products
(when s <= 10) and the squarings into 4 int8 slices (5 for the squarings before the last 8),
with every operand's diagonal split off and added in FP64; it squares E <- 2E + E^2 as three
symmetric products Er^2, Ei^2, (Er + Ei)^2 and solves the Pade step by Newton-Schulz (early
steps at 3 slices).  Smaller walks take the plain form's schedule.  Checked here against the
FP64 eigendecomposition propagator, with the tolerances of the parity tests (complex64 U within
1e-5 relative, states at infidelity <= 1e-10); the per-squaring unitarity residual
(FX_OPT_DRIFT) against one computed directly from the returned U; and the reduced-slice
squarings themselves, by running every squaring at 4 or at 3 slices and comparing the error
with the slices' resolution.
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

C64_REL = 1e-5
INFID = 1e-10


def _dense(n, t=4.5, seed=11):
    """Dense G(n, 0.5) Laplacian walk generator and its FP64 propagator (torch eigh on the
    device: numpy's takes too long at n = 4096)."""
    import torch
    from fastctqw_b200 import graphs
    A = graphs.erdos_renyi(n, 0.5, seed=seed, dtype=np.float32)
    L = np.diag(A.sum(axis=1)) - A
    X = np.asarray(-1j * (-1.0 * L) * t, dtype=np.complex64)
    lam, V = torch.linalg.eigh(torch.from_numpy(X.imag.astype(np.float64)).to("cuda"))
    Vc = V.to(torch.complex128)
    return X, ((Vc * torch.exp(1j * lam)) @ Vc.T).cpu().numpy()


def _walk(X, form, **kw):
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
    e.configure(form=form, **kw)
    e.walk_device(dX, p0, dp, dU)
    torch.cuda.synchronize()
    out = (dU.cpu().numpy(), dp.cpu().numpy(), e.stats(), e.unitarity_drift())
    e.close()
    return out


@pytest.mark.parametrize("n", [1024, 2048, 4096])
def test_mixed_form_meets_the_accuracy_bar(n):
    """Below 4096 the mixed form runs the plain schedule, from 4096 its reduced slices."""
    from fastctqw_b200 import graphs
    X, Uref = _dense(n)
    U, psi, st, _ = _walk(X, "mixed")
    assert st["form"] == 1 and st["structured"] == 1
    assert eo.rel_error(U, Uref) <= C64_REL, eo.rel_error(U, Uref)
    assert eo.infidelity(psi, Uref[:, 0]) <= INFID
    for p0 in (graphs.uniform_state(n), graphs.random_state(n, 3)):
        p = p0.astype(np.complex128)
        assert eo.infidelity(U.astype(np.complex128) @ p, Uref @ p) <= INFID


def test_drift_curve_matches_the_returned_propagator():
    """The residual after the last squaring equals ||U^H U - I||_F / sqrt(n) of the returned U up
    to its complex64 rounding; one value per squaring plus the Pade result."""
    n = 4096
    X, _ = _dense(n)
    for form in ("plain", "mixed"):
        U, _, st, drift = _walk(X, form, drift=True)
        assert len(drift) == st["s"] + 1, (form, drift, st["s"])
        assert all(np.isfinite(drift)) and max(drift) < 1e-4, drift
        U128 = U.astype(np.complex128)
        direct = eo.unitarity_residual(U128)
        # complex64 storage adds ~1e-7 per entry: compare above that floor
        assert abs(drift[-1] - direct) <= 0.5 * direct + 3e-7, (form, drift[-1], direct)


@pytest.mark.parametrize("slices", [4, 3])
def test_reduced_slice_squarings_have_the_slices_resolution(slices):
    """Every squaring at 4 (or 3) slices: the products are right (not garbage) and their error is
    of the size the slices resolve, far above the 5-slice error."""
    n = 4096
    X, Uref = _dense(n, t=2.0)
    U5, _, st, _ = _walk(X, "mixed", sq_n4=0, sq_n3=0)
    kw = {"sq_n4": 64, "sq_n3": 0} if slices == 4 else {"sq_n4": 0, "sq_n3": 64}
    Ur, _, _, _ = _walk(X, "mixed", **kw)
    e5, er = eo.rel_error(U5, Uref), eo.rel_error(Ur, Uref)
    assert e5 <= C64_REL
    bound = {4: 1e-5, 3: 1e-2}[slices]
    assert er <= bound, (slices, er, st["s"])
    # the reduced slices did run: their error is not the 5-slice error
    assert er > e5, (slices, er, e5)


def test_mixed_batch_matches_plain_batch():
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import WalkBatch
    specs = graphs.uneven_batch(12, seed=9, nmin=96, nmax=700)
    Xs = [np.asarray(1j * sp.adjacency(np.float32) * np.float32(sp.t), dtype=np.complex64) for sp in specs]
    P0 = [graphs.random_state(X.shape[0], k) for k, X in enumerate(Xs)]
    ns = [X.shape[0] for X in Xs]
    with WalkBatch(ns) as bp, WalkBatch(ns, form="mixed") as bm:
        a = bp.run(Xs, P0)
        b = bm.run(Xs, P0)
    for k, X in enumerate(Xs):
        lam, V = np.linalg.eigh(X.imag.astype(np.float64))
        ref = V @ (np.exp(1j * lam) * (V.T @ P0[k].astype(np.complex128)))
        assert eo.infidelity(b[k], ref) <= INFID, (k, ns[k])
        assert eo.infidelity(a[k], ref) <= INFID, (k, ns[k])


def test_estimated_selection_uses_the_lanczos_radius():
    """Selector 3: the phase bound of the Pade approximant evaluated at the Lanczos estimate of
    the spectral radius (+10%) instead of the rigorous norm bound.  On the dense Laplacian family
    the estimate is within a few percent of the exact radius (below it, as Ritz values are), the
    selection takes fewer squarings than the Al-Mohy & Higham choice, and the result still meets
    the accuracy bar."""
    from fastctqw_b200 import graphs
    from fastctqw_b200._native import Engine
    import torch
    n = 2048
    X, Uref = _dense(n)
    # exact radius of the shifted generator (trace and rank-one shifts, as the engine applies)
    B = X.imag.astype(np.float64)
    Y = B - np.trace(B) / n * np.eye(n)
    Y -= Y.sum() / n * np.ones((n, n)) / n
    rho = np.abs(np.linalg.eigvalsh(Y)).max()
    _, _, st0, _ = _walk(X, "plain")
    U, psi, st3, _ = _walk(X, "plain", selector="estimated")
    assert st3["sel_outcome"] == 3 and st3["s"] < st0["s"], (st0["s"], st3["s"])
    assert eo.rel_error(U, Uref) <= C64_REL
    assert eo.infidelity(psi, Uref[:, 0]) <= INFID
    for p0 in (graphs.uniform_state(n), graphs.random_state(n, 4)):
        p = p0.astype(np.complex128)
        assert eo.infidelity(U.astype(np.complex128) @ p, Uref @ p) <= INFID
    dev = torch.device("cuda", 0)
    e = Engine(n, np.complex64)
    e.configure(selector="estimated")
    dX = torch.from_numpy(X).to(dev)
    p0 = torch.zeros(n, dtype=torch.complex64, device=dev)
    p0[0] = 1.0
    e.walk_device(dX, p0, torch.empty_like(p0))
    sr = e.spectral_radius()
    e.close()
    assert 0.9 * rho <= sr["lanczos"] <= rho * (1 + 1e-9), (sr, rho)
    assert sr["upper_bound"] >= rho * (1 - 1e-9), (sr, rho)
