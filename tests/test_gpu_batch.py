"""Batched walks through the grouped device pipeline (needs a GPU).

Parity bar (as for single walks): every state at infidelity <= 1e-10 against the FP64 expm of
the same (rounded) generator, (m, s) identical to the per-walk engine's, and the states equal to
the per-walk engine's to 1e-5 (relative, 2-norm).
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

INFID = 1e-10


def _family(count, seed, nmin, nmax, tmin=0.5, tmax=50.0, dtype=np.complex64):
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import walk_generator
    specs = graphs.uneven_batch(count, seed=seed, nmin=nmin, nmax=nmax, tmin=tmin, tmax=tmax)
    Xs, p0 = [], []
    for k, sp in enumerate(specs):
        A = sp.adjacency(np.float64)
        Xs.append(walk_generator(A, sp.t, dtype=dtype))
        n = sp.n
        if k % 3 == 0:
            p0.append(graphs.uniform_state(n).astype(dtype))
        elif k % 3 == 1:
            p0.append(graphs.basis_state(n, k % n).astype(dtype))
        else:
            p0.append(graphs.random_state(n, k).astype(dtype))
    return specs, Xs, p0


@pytest.mark.parametrize("cdtype", [np.complex64, np.complex128])
def test_batch_matches_oracle_and_single_walk_engine(cdtype):
    dtype = cdtype
    from fastctqw_b200.batch import WalkBatch
    from fastctqw_b200._native import Engine
    specs, Xs, p0 = _family(14, seed=5, nmin=20, nmax=420, dtype=dtype)
    b = WalkBatch([X.shape[0] for X in Xs], dtype)
    psis = b.run(Xs, p0)
    m, s = b.selection()
    for k, (X, psi0, psi) in enumerate(zip(Xs, p0, psis)):
        ref = eo.expm(X.astype(np.complex128)) @ psi0.astype(np.complex128)
        inf = eo.infidelity(psi, ref)
        assert inf <= INFID, (k, specs[k], inf, m[k], s[k])
        e = Engine(X.shape[0], dtype)
        e.configure(form="plain")   # the batch's product arithmetic (int8 slices, FP64 masters)
        single = e.walk_host(X, psi0)
        st = e.stats()
        e.close()
        assert (m[k], s[k]) == (st["m"], st["s"]), (k, specs[k])
        assert np.linalg.norm(psi - single) <= 1e-5 * np.linalg.norm(single), k


def test_batch_graph_and_eager_agree_bitwise():
    from fastctqw_b200.batch import WalkBatch
    _, Xs, p0 = _family(9, seed=8, nmin=100, nmax=300)
    ns = [X.shape[0] for X in Xs]
    a = WalkBatch(ns).run(Xs, p0)
    b = WalkBatch(ns, graph=False).run(Xs, p0)
    c = WalkBatch(ns).run(Xs, p0)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y) and np.array_equal(x, z)


def test_batch_small_norms_use_low_pade_degrees():
    from fastctqw_b200.batch import WalkBatch
    _, Xs, p0 = _family(10, seed=9, nmin=16, nmax=200, tmin=0.001, tmax=0.3)
    b = WalkBatch([X.shape[0] for X in Xs])
    psis = b.run(Xs, p0)
    m, s = b.selection()
    assert set(m.tolist()) - {13}, m      # some walks take m < 13
    for X, psi0, psi in zip(Xs, p0, psis):
        ref = eo.expm(X.astype(np.complex128)) @ psi0.astype(np.complex128)
        assert eo.infidelity(psi, ref) <= INFID


def test_batch_rejects_general_generators():
    from fastctqw_b200.batch import WalkBatch
    rng = np.random.default_rng(1)
    X = (rng.standard_normal((40, 40)) + 1j * rng.standard_normal((40, 40))).astype(np.complex64)
    b = WalkBatch([40])
    with pytest.raises(ValueError):
        b.run([X], [np.ones(40, np.complex64) / np.sqrt(40)])


def test_large_scaling_walks_keep_double_level_accuracy():
    """Walks with many squarings (G(n, p) adjacency, no rank-one shift, s ~ 10-11) amplify any
    systematic bias of the int8 products: the slice digits must be symmetric about zero
    (a bias of -1/2 per digit once cost three orders of magnitude here).  Bar: 5e-12."""
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import WalkBatch
    Xs, p0, refs = [], [], []
    for n, p, t, seed in ((1536, 0.45, 6.81, 11), (1280, 0.21, 5.22, 12)):
        A = graphs.erdos_renyi(n, p, seed=seed, dtype=np.float64)
        t32 = float(np.float32(t))
        Xs.append(np.asarray(1j * A * t32, dtype=np.complex64))
        psi0 = graphs.uniform_state(n)
        p0.append(psi0)
        lam, V = np.linalg.eigh(A)
        refs.append(V @ (np.exp(1j * lam * t32) * (V.T @ psi0.astype(np.complex128))))
    b = WalkBatch([X.shape[0] for X in Xs])
    psis = b.run(Xs, p0)
    m, s = b.selection()
    for k in range(len(Xs)):
        assert s[k] >= 9, (m, s)
        assert eo.infidelity(psis[k], refs[k]) <= 5e-12, (k, eo.infidelity(psis[k], refs[k]), s[k])


def test_autotuned_schedule_keeps_the_states_bitwise():
    """The autotuner times the candidate schedules of the post-selection products on the batch
    and keeps the fastest; a schedule orders the tiles, never changes their arithmetic."""
    from fastctqw_b200.batch import WalkBatch
    _, Xs, p0 = _family(12, seed=10, nmin=64, nmax=600)
    ns = [X.shape[0] for X in Xs]
    ref = WalkBatch(ns).run(Xs, p0)
    b = WalkBatch(ns, autotune=True)
    got = b.run(Xs, p0)
    sch = b.schedule()
    assert len(sch["tuned"]) == 5 and all(ms > 0 for _, _, ms in sch["tuned"])
    best = min(sch["tuned"], key=lambda r: r[2])
    assert (sch["tile_group"], sch["tile_order"]) == best[:2]
    again = b.run(Xs, p0)                  # the kept schedule, no tuning
    c = WalkBatch(ns)
    c.set_schedule(16, 1)
    other = c.run(Xs, p0)
    for x, y, z, w in zip(ref, got, again, other):
        assert np.array_equal(x, y) and np.array_equal(x, z) and np.array_equal(x, w)
