"""Long-time walks (needs a GPU): generators whose selections take 12 to 17 squarings.

Seeded walks of the selector's generator family (random regular, G(n, p) and weighted complete
graphs, adjacency or Laplacian, t log-uniform up to 1000), the ones whose results are the most
sensitive to the accuracy of the Pade step: its error is amplified 2^s by the squarings.  The
state psi0 = (v_max + v_min) / sqrt 2 (the eigenvectors at the two ends of the spectrum) exposes
a phase error most.  Checked in both forms against the FP64 eigendecomposition at the parity
bar (infidelity <= 1e-10), which needs the diagonal split in the plain form's powers and Pade
products: without it the worst of these walks reached 5.7e-7.
"""
import itertools
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# indices in make_walks(192, seed=3, nmin=64, nmax=2048, tmin=0.1, tmax=1000): the walks with
# the largest errors before the plain form split its Pade products' diagonals
HARD = (12, 21, 29, 34, 82, 93, 110, 117, 127, 136)


def _walks():
    from fastctqw_b200 import selector
    gen = selector.make_walks(192, 3, 64, 2048, 0.1, 1000.0)
    out = []
    for k, (X, meta) in enumerate(itertools.islice(gen, max(HARD) + 1)):
        if k in HARD:
            out.append((X, meta))
    return out


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_long_time_walks_meet_the_bar(form):
    import torch
    from fastctqw_b200.batch import WalkBatch
    dev = torch.device("cuda", 0)
    walks = _walks()
    Xs = [X for X, _ in walks]
    dX = [torch.from_numpy(X).to(dev) for X in Xs]
    p0s, refs = [], []
    for X in Xs:
        lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to(dev))
        p0s.append(((V[:, -1] + V[:, 0]) / math.sqrt(2.0)).to(torch.complex64))
        refs.append((torch.exp(1j * lam[-1]) * V[:, -1] + torch.exp(1j * lam[0]) * V[:, 0]) / math.sqrt(2.0))
    outs = [torch.empty_like(p) for p in p0s]
    with WalkBatch([X.shape[0] for X in Xs], form=form) as b:
        b.run_device(dX, p0s, outs)
        torch.cuda.synchronize()
        _, s = b.selection()
    assert s.min() >= 12, s
    for k, (q, ref) in enumerate(zip(outs, refs)):
        q = q.to(torch.complex128)
        inf = float(1.0 - torch.vdot(ref, q).abs() ** 2 / (torch.vdot(q, q).real * torch.vdot(ref, ref).real))
        assert inf <= 1e-10, (form, walks[k][1], int(s[k]), inf)


def test_regular_laplacian_walk_with_nine_squarings():
    """A 3-regular Laplacian walk (N = 2784, graph seed 2034370348, t = 583.08..., the selector
    family's generator; 9 squarings) on which the exact complex square reached 2.6e-9: its
    iterates' dominant diagonal costs the unsplit slices their bits, and the chain amplifies
    that 2^9.  Both forms now square it as three split products."""
    import torch
    from fastctqw_b200 import graphs
    from fastctqw_b200.batch import WalkBatch
    dev = torch.device("cuda", 0)
    n, d, gseed, t = 2784, 3, 2034370348, 583.0815413536579
    A = graphs.random_regular(n, d, gseed, np.float64)
    X = np.asarray(-1j * (-(np.diag(A.sum(axis=1)) - A)) * t, dtype=np.complex64)
    lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to(dev))
    Vc = V.to(torch.complex128)
    for form in ("plain", "mixed"):
        for a, b in ((0, -1), (0, 1), (-2, -1)):   # pairs of eigenvectors at the spectrum's ends
            p0 = (V[:, a] + V[:, b]) / math.sqrt(2.0)
            ref = Vc @ (torch.exp(1j * lam) * (Vc.T @ p0.to(torch.complex128)))
            out = [torch.empty(n, dtype=torch.complex64, device=dev)]
            with WalkBatch([n], form=form) as bt:
                bt.run_device([torch.from_numpy(X).to(dev)], [p0.to(torch.complex64)], out)
                torch.cuda.synchronize()
                _, s = bt.selection()
            q = out[0].to(torch.complex128)
            inf = float(1.0 - torch.vdot(ref, q).abs() ** 2 / (torch.vdot(q, q).real * torch.vdot(ref, ref).real))
            assert inf <= 1e-10, (form, a, b, int(s[0]), inf)

