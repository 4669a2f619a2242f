"""Device-side set-up and read-out of walks (needs a GPU): X built from an edge list, the
Hermitian check, the propagator step, probabilities, adjacency-list walks and time curves.

Bars: the device-built X equals the host-built X of the reference's numpy expressions bit for
bit; the Hermitian check agrees with np.allclose; the GEMV within 1e-6 (complex64) / 1e-13
(complex128) relative of numpy in FP64; probabilities exact in FP64 of the stored amplitudes;
time-curve probabilities against the FP64 propagator of the generator as rounded in the walk's
dtype: one walk per time ("batch") within 1e-6 (complex64: the states are stored in complex64)
and 1e-9 (complex128) absolute; a stepped propagator (20 steps, U stored in the walk's dtype)
within 1e-5 and 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(n, p, seed, loops=0):
    rng = np.random.default_rng(seed)
    A = np.triu(rng.random((n, n)) < p, 1)
    A = (A | A.T).astype(np.float64)
    for v in rng.choice(n, loops, replace=False):
        A[v, v] = 1.0
    return A


def _edges(A, dup=True):
    u, v = np.nonzero(np.triu(A))
    e = np.stack([u, v], 1).astype(np.int64)
    if dup and len(e):
        e = np.concatenate([e, e[: len(e) // 3, ::-1]])   # repeated edges, both directions
    return e


def _host_X(A, t, gamma, laplacian, cdtype):
    """-1j * H * t exactly as FastCTQW/Operator.py:49-56 computes it (numpy, in cdtype)."""
    if laplacian:
        H = -gamma * np.asarray(np.diag(A.sum(axis=1)) - A, dtype=cdtype)
    else:
        H = -gamma * np.asarray(A, cdtype)
    return np.asarray(-1j * H * t, dtype=cdtype)


@pytest.mark.parametrize("laplacian", [False, True])
@pytest.mark.parametrize("cdtype", [np.complex64, np.complex128])
def test_generator_from_edges_is_bitwise_the_host_matrix(laplacian, cdtype):
    from fastctqw_b200.device import build_generator
    for n, p, seed, t, gamma in ((97, 0.1, 1, 4.5, 1.0), (300, 0.5, 2, 0.37, 0.83), (5, 0.0, 3, 2.0, 1.0)):
        A = _graph(n, p, seed, loops=2)
        X = build_generator(n, _edges(A), t, gamma, laplacian, cdtype).cpu().numpy()
        ref = _host_X(A, t, gamma, laplacian, cdtype)
        assert np.array_equal(X, ref), (n, laplacian, np.abs(X - ref).max())


def test_generator_rejects_bad_edges():
    from fastctqw_b200.device import build_generator
    with pytest.raises(ValueError):
        build_generator(10, np.array([[0, 1], [3, 10]]), 1.0)
    with pytest.raises(ValueError):
        build_generator(10, np.array([[-1, 2]]), 1.0)


@pytest.mark.parametrize("cdtype", [np.complex64, np.complex128, np.float32, np.float64])
def test_hermitian_check_agrees_with_allclose(cdtype):
    import torch
    from fastctqw_b200.device import is_hermitian
    rng = np.random.default_rng(4)
    for n in (1, 31, 33, 130):
        M = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if np.iscomplexobj(np.zeros(1, cdtype)) else 0)
        H = np.asarray((M + M.conj().T) / 2, dtype=cdtype)
        cases = [H]
        if n > 1:
            Hb = H.copy(); Hb[n - 1, 0] += 1e-3; cases.append(Hb)          # asymmetric entry
            Hc = H.copy(); Hc[0, 1] = np.nan; cases.append(Hc)            # NaN fails
            Hd = H.copy(); Hd[1, 0] *= 1 + 1e-7; cases.append(Hd)         # within rtol
        if np.iscomplexobj(H):
            He = H.copy(); He[0, 0] += 1e-2j; cases.append(He)            # complex diagonal
        for K in cases:
            dK = torch.from_numpy(np.ascontiguousarray(K)).cuda()
            assert is_hermitian(dK) == bool(np.allclose(K, K.conj().T)), (n, cdtype)
            if np.iscomplexobj(K):   # X = -iK is skew-Hermitian exactly when K is Hermitian
                X = np.ascontiguousarray(-1j * K).astype(cdtype)
                got = is_hermitian(torch.from_numpy(X).cuda(), skew=True)
                assert got == bool(np.allclose(X, -X.conj().T)), (n, cdtype)


@pytest.mark.parametrize("cdtype,tol", [(np.complex64, 1e-6), (np.complex128, 1e-13)])
def test_propagator_step_and_probabilities(cdtype, tol):
    import torch
    from fastctqw_b200.device import apply_propagator, probabilities
    rng = np.random.default_rng(5)
    n = 515
    U = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(cdtype)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(cdtype)
    y = apply_propagator(torch.from_numpy(U).cuda(), torch.from_numpy(x).cuda()).cpu().numpy()
    ref = U.astype(np.complex128) @ x.astype(np.complex128)
    assert np.linalg.norm(y - ref) <= tol * np.linalg.norm(ref)
    dx = torch.from_numpy(x).cuda()
    p = probabilities(dx).cpu().numpy()
    x128 = x.astype(np.complex128)
    assert np.array_equal(p, x128.real ** 2 + x128.imag ** 2)
    nodes = [3, 0, n - 1, 3]
    pm = probabilities(dx, nodes).cpu().numpy()
    assert np.array_equal(pm, p[nodes])
    bad = probabilities(dx, [1, n, -1]).cpu().numpy()
    assert bad[0] == p[1] and np.isnan(bad[1]) and np.isnan(bad[2])


def _exact_states(X, psi0, powers=(1,)):
    """exp(k X) psi0 in FP64 for a generator X = i K (K real symmetric), for each k."""
    K = X.imag.astype(np.float64)
    lam, V = np.linalg.eigh(K)
    c = V.T @ psi0.astype(np.complex128)
    return [V @ (np.exp(1j * k * lam) * c) for k in powers]


def test_adjacency_list_walk_matches_the_matrix_walk():
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    A = _graph(200, 0.1, 6)
    adj = [list(np.nonzero(A[u])[0]) for u in range(200)]
    s0 = State.getUniformSuperposition(200)
    w1 = Ctqw.from_adjacency_list(adj, s0, laplacian=True)
    w2 = Ctqw.from_numpy_array(A.astype(np.float32), s0, laplacian=True)
    w1.runWalk(3.3)
    w2.runWalk(3.3)
    assert np.array_equal(w1.getFinalState().getState(), w2.getFinalState().getState())
    op = w1.getOperator()
    op.buildExpmOperator(3.3)
    w2.getOperator().buildExpmOperator(3.3)
    assert np.array_equal(op._expmMat, w2.getOperator()._expmMat)


@pytest.mark.parametrize("wdtype,batch_tol,step_tol", [(np.float32, 1e-6, 1e-5), (np.float64, 1e-9, 1e-8)])
def test_time_curves(wdtype, batch_tol, step_tol):
    """References: the FP64 propagator of the generator as the walk's dtype rounds it (for
    complex64 the rounding of t itself is larger than the algorithm's error)."""
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    cdtype = np.complex64 if wdtype == np.float32 else np.complex128
    n = 160
    A = _graph(n, 0.08, 7)
    adj = [list(np.nonzero(A[u])[0]) for u in range(n)]
    psi0 = np.zeros(n, np.complex64)
    psi0[5] = 1.0
    marks = [5, 17, 80]
    w = Ctqw.from_adjacency_list(adj, State(psi0), dtype=wdtype)
    grid = 0.4 * np.arange(1, 21)
    X1 = _host_X(A, grid[0], 1.0, False, cdtype)
    stepped = np.abs(np.array(_exact_states(X1, psi0, range(1, 21)))) ** 2
    steps = w.runWalks(grid, marks)                      # uniform grid: stepped propagator
    assert steps.shape == (20, 3)
    assert np.abs(steps - stepped[:, marks]).max() <= step_tol, np.abs(steps - stepped[:, marks]).max()
    exact = np.array([np.abs(_exact_states(_host_X(A, t, 1.0, False, cdtype), psi0)[0]) ** 2 for t in grid])
    batch = w.runWalks(grid, marks, method="batch")      # one walk per time
    assert np.abs(batch - exact[:, marks]).max() <= batch_tol, np.abs(batch - exact[:, marks]).max()
    odd = np.array([0.05, 1.7, 3.1, 9.0])
    got = w.runWalks(odd)                                # not uniform: batch, all nodes
    assert got.shape == (4, n)
    ref = np.array([np.abs(_exact_states(_host_X(A, t, 1.0, False, cdtype), psi0)[0]) ** 2 for t in odd])
    assert np.abs(got - ref).max() <= batch_tol, np.abs(got - ref).max()
    last = w.getFinalState().getState().astype(np.complex128)
    assert np.allclose(np.abs(last) ** 2, got[-1], atol=1e-6)
