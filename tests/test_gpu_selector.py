"""Learned (m, s) selector on the GPU: kernels against the CPU oracle, training, and what the
trained network gains over the plain Al-Mohy & Higham selection (needs a GPU).

Tolerances: loss and gradient of the FP32 fused kernel within 1e-4 (relative) of the FP64
oracle; BF16 inference within 3e-2 of the FP64 forward pass; walks at infidelity <= 1e-10
against the FP64 eigendecomposition.
"""
import os

import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _t(a, dtype):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def test_fused_forward_backward_matches_oracle():
    import torch
    from fastctqw_b200 import _native, selector
    rng = np.random.default_rng(1)
    w = selector.init_weights(7) + (0.05 * rng.standard_normal(5126)).astype(np.float32)
    x = rng.standard_normal((150, 8)).astype(np.float32)
    ym = rng.integers(0, 5, 150).astype(np.int32)
    ys = (rng.random(150) * 12).astype(np.float32)
    g = torch.zeros(5126, device="cuda")
    loss = torch.zeros(1, device="cuda")
    # device copies held in names: a temporary's memory may be reused before the call runs
    dw, dx, dym, dys = _t(w, torch.float32), _t(x, torch.float32), _t(ym, torch.int32), _t(ys, torch.float32)
    rc = _native.lib().fx_mlp_loss_grad(dw.data_ptr(), dx.data_ptr(), dym.data_ptr(), dys.data_ptr(), 150,
                                        0.25, g.data_ptr(), loss.data_ptr(), None)
    assert rc == 0, _native.lib().fx_mlp_error()
    l_ref, g_ref = mo.loss_grad(w.astype(np.float64), x.astype(np.float64), ym, ys.astype(np.float64), 0.25)
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * abs(l_ref)
    gd = g.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(gd - g_ref) <= 1e-4 * np.linalg.norm(g_ref)


def test_bf16_inference_matches_oracle():
    from fastctqw_b200 import selector
    rng = np.random.default_rng(2)
    w = selector.init_weights(4)
    x = rng.standard_normal((333, 8)).astype(np.float32)
    out = selector.infer(w, x)
    ref = mo.forward(w.astype(np.float64), x.astype(np.float64))[0]
    assert np.linalg.norm(out - ref) <= 3e-2 * np.linalg.norm(ref)


def test_training_on_the_device_fits_a_rule():
    """Labels from a fixed rule of the features; the device training must learn it."""
    from fastctqw_b200 import selector
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2048, 8)).astype(np.float32)
    cls = np.digitize(x[:, 1] + 0.5 * x[:, 6], [-1.0, -0.3, 0.3, 1.0]).astype(np.int32)
    m = np.array([selector.DEGREES[c] for c in cls])
    s = np.clip(np.rint(4 + 2 * x[:, 7]), 0, None).astype(np.int32)
    ds = {"features": x, "cert_m": m, "cert_s": s}
    w, losses = selector.train(ds, epochs=60, batch=128, lr=3e-3)
    assert losses[-1] < 0.25 * losses[0], losses[[0, -1]]
    pm, ps = selector.proposals(selector.infer(w, x))
    assert np.mean(pm == m) > 0.9 and np.mean(ps == s) > 0.8


def _walks(count, seed):
    from fastctqw_b200 import selector
    walks = list(selector.make_walks(count, seed, 48, 320, 0.2, 200.0))
    Xs = [X for X, _ in walks]
    psi0 = []
    for k, X in enumerate(Xs):
        p = np.zeros(X.shape[0], np.complex64)
        p[k % X.shape[0]] = 1
        psi0.append(p)
    refs = []
    for X, p in zip(Xs, psi0):
        lam, V = np.linalg.eigh((X.astype(np.complex128) / 1j).real)
        refs.append(V @ (np.exp(1j * lam) * (V.T @ p.astype(np.complex128))))
    return Xs, psi0, refs


def _inf(a, b):
    a = a.astype(np.complex128)
    return 1 - abs(np.vdot(b, a)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def test_certified_selection_is_cheaper_and_accurate():
    from fastctqw_b200.batch import WalkBatch
    Xs, psi0, refs = _walks(20, 11)
    b = WalkBatch([X.shape[0] for X in Xs], selector="certified")
    psis = b.run(Xs, psi0)
    m, s = b.selection()
    d = b.details()
    assert (d["outcome"] == 1).sum() > 0
    for k in range(len(Xs)):
        assert _inf(psis[k], refs[k]) <= 1e-10, k
    assert s.sum() < d["plain_s"].sum()


def test_trained_selector_gains_over_plain():
    """The shipped network: the learned selection never costs more products than the estimated
    one it falls back to, saves squarings over the plain selection, and every walk stays at
    infidelity <= 1e-10; walks on the plain choice give the plain result bit for bit."""
    from fastctqw_b200 import selector
    from fastctqw_b200.batch import WalkBatch
    assert os.path.exists(selector.WEIGHTS)
    selector.set_weights()
    Xs, psi0, refs = _walks(24, 12)
    ns = [X.shape[0] for X in Xs]
    bp = WalkBatch(ns)
    plain = bp.run(Xs, psi0)
    m_plain, s_plain = bp.selection()
    be = WalkBatch(ns, selector="estimated")
    be.run(Xs, psi0)
    m_est, s_est = be.selection()
    bl = WalkBatch(ns, selector="learned")
    learned = bl.run(Xs, psi0)
    m_l, s_l = bl.selection()
    d = bl.details()
    cost = lambda m, s: np.array([selector.PRODUCTS[int(a)] + int(b) for a, b in zip(m, s)])
    assert np.all(cost(m_l, s_l) <= cost(m_est, s_est)), (m_l, s_l, m_est, s_est)
    assert s_l.sum() < s_plain.sum(), (s_l.sum(), s_plain.sum())
    for k in range(len(Xs)):
        assert _inf(learned[k], refs[k]) <= 1e-10, (k, _inf(learned[k], refs[k]))
        # a walk left on its fallback choice with the plain run's (m, s) computes the same
        # (the fallback of these selections comes from norm bounds, not the 1-norm estimates,
        # so it can take a squaring more than the plain selection)
        if d["outcome"][k] <= 0 and (m_l[k], s_l[k]) == (m_plain[k], s_plain[k]):
            assert np.array_equal(learned[k], plain[k])


def test_rejected_proposals_fall_back_to_the_estimated_choice():
    """A network that always proposes (13, 0) is rejected by the bound for every walk that
    needs squarings; those walks then run the estimated selection's (m, s) (or the plain one
    where nothing is cheaper), and the whole batch equals the estimated run bit for bit."""
    from fastctqw_b200 import selector
    from fastctqw_b200.batch import WalkBatch
    w = np.zeros(5126, np.float32)
    w[-6 + 4] = 10.0          # logit of m = 13; s output 0
    selector.set_weights(w)
    Xs, psi0, _ = _walks(10, 13)
    ns = [X.shape[0] for X in Xs]
    be = WalkBatch(ns, selector="estimated")
    est = be.run(Xs, psi0)
    bl = WalkBatch(ns, selector="learned")
    learned = bl.run(Xs, psi0)
    d = bl.details()
    need = d["plain_s"] > 0
    assert need.any()
    assert np.all(np.isin(d["outcome"][need], (3, -1)))
    assert np.array_equal(np.stack(bl.selection()), np.stack(be.selection()))
    for k in range(len(Xs)):
        assert np.array_equal(learned[k], est[k])
    if os.path.exists(selector.WEIGHTS):
        selector.set_weights()     # restore the shipped weights for later tests


def test_mixed_degree_batches_twice():
    """Certified choices mix every Pade degree, scaled or not, in one batch; a second run on
    the same workspace must give the same states (no term may read another run's data)."""
    from fastctqw_b200 import selector
    from fastctqw_b200.batch import WalkBatch
    walks = list(selector.make_walks(40, 21, 32, 256, 0.001, 100.0))
    Xs = [X for X, _ in walks]
    b = WalkBatch([X.shape[0] for X in Xs], selector="certified")
    first = b.run(Xs)
    m, s = b.selection()
    assert len(set(m.tolist())) >= 3, m
    second = b.run(Xs)
    for k, X in enumerate(Xs):
        lam, V = np.linalg.eigh((X.astype(np.complex128) / 1j).real)
        p0 = np.full(X.shape[0], 1 / np.sqrt(X.shape[0]))
        ref = V @ (np.exp(1j * lam) * (V.T @ p0))
        assert _inf(first[k], ref) <= 1e-10, (k, m[k], s[k])
        assert np.array_equal(first[k], second[k])


def test_sampled_plain_comparison_checks_non_plain_walks():
    """After a learned run, the smallest walks that took a non-plain (m, s) are re-run with the
    plain (m, s) and compared; on sound proposals the states agree to far below 1e-10."""
    from fastctqw_b200 import selector
    from fastctqw_b200.batch import OPT_SAMPLE_WALKS, WalkBatch
    selector.set_weights()
    Xs, psi0, refs = _walks(16, 14)
    ns = [X.shape[0] for X in Xs]
    b = WalkBatch(ns, selector="learned")
    b.run(Xs, psi0)
    d = b.details()
    m, s = b.selection()
    nonplain = sorted(ns[k] for k in np.nonzero((m != d["plain_m"]) | (s != d["plain_s"]))[0])

    def expected(k):   # the smallest non-plain walks, dropped largest-first to a tenth of the
        pick = nonplain[:k]   # batch by N^3, but never fewer than one
        while len(pick) > 1 and sum(n ** 3 for n in pick) > 0.1 * sum(n ** 3 for n in ns):
            pick = pick[:-1]
        return len(pick)

    assert expected(2) > 0, nonplain
    chk = b.sample_check()
    assert chk["sampled"] == expected(2), (chk, nonplain)
    assert chk["max_infidelity"] <= 1e-10
    b.set_option(OPT_SAMPLE_WALKS, 5)
    b.run(Xs, psi0)
    assert b.sample_check()["sampled"] == expected(5)
    one = WalkBatch([ns[0]], selector="learned")     # a batch of one: never re-run
    one.run([Xs[0]], [psi0[0]])
    d1 = one.details()
    m1, s1 = one.selection()
    non_plain_one = bool(m1[0] != d1["plain_m"][0] or s1[0] != d1["plain_s"][0])
    # skipped (-1) when the single walk took a non-plain (m, s); nothing to compare (0) otherwise
    assert one.sample_check()["sampled"] == (-1 if non_plain_one else 0)
