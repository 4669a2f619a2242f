"""Parity on the benchmark workloads themselves (needs a GPU).

* The small plain-method walk: networkx random 4-regular graph, N = 1024 (seeded), H = -A
  (the reference's Operator convention, FastCTQW/Operator.py:49-56), t = 4.5, built through
  ``Ctqw.from_networkx_graph`` (FastCTQW/Ctqw.py:45-57, the entry point of the reference's
  README).  The uniform superposition is an eigenvector of every regular graph, so it alone
  would be a near-vacuous check: the basis state |0> and a seeded random state are run too,
  and the full U is compared.
* The dense walk family at N = 2048 and 4096: G(n, 0.5) Laplacian, t = 4.5, the family of the
  N = 10000 benchmark walk.

Tolerances: complex64 U within 1e-5 relative (Frobenius) of the FP64 propagator, states at
infidelity <= 1e-10.  The FP64 oracle is the eigendecomposition propagator
V diag(exp(-i lambda t)) V^T of the real symmetric H (numpy on the host at N = 1024, torch FP64
on the device above), the most accurate reference for these inputs.
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

C64_REL = 1e-5
INFID = 1e-10
T = 4.5


def _states(n, seed):
    from fastctqw_b200 import graphs
    return {"uniform": graphs.uniform_state(n), "e0": graphs.basis_state(n, 0),
            "random": graphs.random_state(n, seed)}


def test_regular_graph_walk_n1024_through_networkx_entry_point():
    import networkx as nx
    from fastctqw_b200 import fastexpm
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    n = 1024
    G = nx.random_regular_graph(4, n, seed=1024)
    A = nx.to_numpy_array(G, dtype=np.float32, nodelist=range(n))
    H = eo.build_hamiltonian(A, 1.0, False, dtype=np.float64).real      # H = -A
    lam, V = np.linalg.eigh(H)
    U_ref = (V * np.exp(-1j * lam * T)) @ V.T
    # full U through the drop-in (X = -1j H t in complex64, as Operator._buildUnitory forms it)
    X = np.asarray(-1j * (-1.0 * A.astype(np.complex64)) * T, dtype=np.complex64)
    with fastexpm.ExpMatComplex64(n) as e:
        U = e.run(X)
    assert eo.rel_error(U, U_ref) <= C64_REL, eo.rel_error(U, U_ref)
    # states through Ctqw.from_networkx_graph
    for kind, p0 in _states(n, 7).items():
        w = Ctqw.from_networkx_graph(G, State(p0))
        w.runWalk(T)
        psi = w.getFinalState().getState()
        inf = eo.infidelity(psi, U_ref @ p0.astype(np.complex128))
        assert inf <= INFID, (kind, inf)
        w.free()


def test_networkx_entry_point_equals_matrix_entry_point(golden):
    """from_networkx_graph(G) runs the same walk as the ndarray constructor on
    nx.to_numpy_array(G, float32) (FastCTQW/Ctqw.py:57), bit for bit, on the golden graphs."""
    import networkx as nx
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    done = 0
    for name, c in golden.items():
        if "psi_ref_e0" not in c or c["A"].dtype != np.float32:
            continue
        A = c["A"]
        G = nx.from_numpy_array(A.astype(np.float64))
        gamma, lap, t = float(c["gamma"]), bool(c["laplacian"]), float(c["t"])
        p0 = c["psi0_random"]
        a = Ctqw.from_networkx_graph(G, State(p0), gamma, lap)
        b = Ctqw(A, State(p0), gamma, lap)
        a.runWalk(t)
        b.runWalk(t)
        assert np.array_equal(a.getFinalState().getState(), b.getFinalState().getState()), name
        a.free()
        b.free()
        done += 1
    assert done >= 3


@pytest.mark.parametrize("n", [2048, 4096])
def test_dense_laplacian_walk_full_u(n):
    import torch
    from fastctqw_b200 import fastexpm, graphs
    A = graphs.erdos_renyi(n, 0.5, seed=2024 + n, dtype=np.float32)
    L = np.diag(A.sum(axis=1)) - A
    X = np.asarray(-1j * (-1.0 * L) * T, dtype=np.complex64)     # H = -(D - A), X = -1j H t
    with fastexpm.ExpMatComplex64(n) as e:
        U = e.run(X)
        st = e.stats()
    dev = torch.device("cuda", 0)
    lam, V = torch.linalg.eigh(torch.from_numpy(-L.astype(np.float64)).to(dev))
    Vc = V.to(torch.complex128)
    U_ref = (Vc * torch.exp(-1j * lam * T)) @ Vc.T
    Ud = torch.from_numpy(U).to(dev).to(torch.complex128)
    rel = float(torch.linalg.matrix_norm(Ud - U_ref) / torch.linalg.matrix_norm(U_ref))
    assert rel <= C64_REL, (n, rel, st["m"], st["s"])
    for kind, p0 in _states(n, n).items():
        p = torch.from_numpy(p0).to(dev).to(torch.complex128)
        ref = (U_ref @ p).cpu().numpy()
        psi = (Ud @ p).cpu().numpy()
        inf = eo.infidelity(psi, ref)
        assert inf <= INFID, (n, kind, inf)
