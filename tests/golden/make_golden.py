"""Generate the golden fixtures from the reference's own CPU path.

Run where a checkout of the reference exists (it is read, never modified), passing its root
directory as the argument or in the environment variable FASTCTQW_REFERENCE_ROOT:

    python tests/golden/make_golden.py <reference checkout>

The reference package ``FastCTQW`` imports matplotlib/seaborn eagerly
(FastCTQW/__init__.py:3 via Plot.py:1-2) and the compiled ``_fastexpm_core``
(FastCTQW/fastexpm/_wrapper.py:6); neither is needed by its CPU path, so both are stubbed.
Every fixture records the inputs and the outputs of:

* ``Operator(A, gamma, laplacian, device="cpu").buildExpmOperator(t)``
  (FastCTQW/Operator.py:70-78) -> ``U_ref`` (the reference's scipy.linalg.expm result),
* ``Ctqw(A, State(psi0), gamma, laplacian).runWalk(t)`` (FastCTQW/Ctqw.py:90-94) ->
  ``psi_ref``,
* for the reference test families (tests/test_fastexpm_accuracy.py:83-160: complete,
  G(N, 0.05), random 4-regular, each exponentiated as ``1j*A``): scipy.linalg.expm, which
  is what the reference's CPU Operator calls, and the reference test's own Taylor oracle
  ``matrix_exp_taylor`` (tests/test_fastexpm_accuracy.py:10-56),
* for its perf-test inputs ``A_real + 1j*rand`` (tests/test_fastexpm_perf.py:11-61):
  scipy.linalg.expm,
plus an FP64 eigendecomposition propagator where H is Hermitian.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _stub_reference_imports():
    for name in ["matplotlib", "matplotlib.pyplot", "matplotlib.ticker", "seaborn"]:
        mod = types.ModuleType(name)
        sys.modules[name] = mod
    sys.modules["matplotlib.ticker"].ScalarFormatter = object
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    core = types.ModuleType("FastCTQW.fastexpm._fastexpm_core")
    sys.modules["FastCTQW.fastexpm._fastexpm_core"] = core


def load_reference(ref_root: str):
    _stub_reference_imports()
    sys.path.insert(0, ref_root)
    import FastCTQW  # noqa: F401
    from FastCTQW.Ctqw import Ctqw
    from FastCTQW.Operator import Operator
    from FastCTQW.State import State
    spec = importlib.util.spec_from_file_location(
        "ref_test_fastexpm_accuracy", os.path.join(ref_root, "tests", "test_fastexpm_accuracy.py"))
    tmod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tmod)
    return Ctqw, Operator, State, tmod.matrix_exp_taylor


def main(ref_root: str):
    sys.path.insert(0, REPO)
    from fastctqw_b200 import graphs
    Ctqw, Operator, State, taylor = load_reference(ref_root)
    import scipy.linalg as sl

    cases = {}
    meta = {}

    def walk_case(name, A, t, gamma=1.0, lap=False, psi_kinds=("uniform", "e0", "random"),
                  keep_u=True):
        n = A.shape[0]
        op = Operator(A, gamma, lap, "cpu")
        op.buildExpmOperator(t)
        U_ref = op.getOperator()
        H = np.asarray(op._hamiltonian, dtype=np.complex128)
        lam, V = np.linalg.eigh(H)
        U_eig = (V * np.exp(-1j * lam * t)) @ V.conj().T
        entry = {"A": A, "t": np.float64(t), "gamma": np.float64(gamma),
                 "laplacian": np.int8(lap)}
        if keep_u:
            entry["U_ref"] = U_ref
            entry["U_eig"] = U_eig
        for kind in psi_kinds:
            if kind == "uniform":
                st = State.getUniformSuperposition(n)
            elif kind == "e0":
                st = State.getSingleNodeState(n, 0)
            else:
                st = State(graphs.random_state(n, 7))
            w = Ctqw(A, st, gamma, lap)
            w.runWalk(t)
            entry[f"psi0_{kind}"] = st.getState()
            entry[f"psi_ref_{kind}"] = w.getFinalState().getState()
            entry[f"psi_eig_{kind}"] = U_eig @ st.getState().astype(np.complex128)
        cases[name] = entry
        meta[name] = {"kind": "walk", "n": n, "t": t, "gamma": gamma, "laplacian": lap,
                      "dtype": str(A.dtype)}

    # Configuration families at sizes the CPU finishes in seconds.
    walk_case("reg4_n64", graphs.random_regular(64, 4, seed=11), 4.5)
    walk_case("reg4_n128", graphs.random_regular(128, 4, seed=12), 4.5)
    walk_case("reg4_n200_f64", graphs.random_regular(200, 4, seed=13, dtype=np.float64), 4.5,
              keep_u=False)
    walk_case("erlap_n64", graphs.erdos_renyi(64, 0.5, seed=21), 4.5, lap=True)
    walk_case("erlap_n96_f64", graphs.erdos_renyi(96, 0.5, seed=22, dtype=np.float64), 4.5,
              lap=True)
    walk_case("erlap_n256", graphs.erdos_renyi(256, 0.5, seed=23), 4.5, lap=True,
              keep_u=False)
    walk_case("er_adj_n77", graphs.erdos_renyi(77, 0.2, seed=31), 3.3)
    walk_case("reg7_n50_t20", graphs.random_regular(50, 7, seed=32), 20.0, gamma=0.5)
    walk_case("wlap_n48_t100", graphs.weighted_complete(48, seed=51), 100.0, lap=True)
    walk_case("wlap_n48_t100_f64", graphs.weighted_complete(48, seed=52, dtype=np.float64),
              100.0, lap=True)
    walk_case("er_adj_n3", graphs.erdos_renyi(3, 0.9, seed=4), 1.0)
    walk_case("single_n1", np.zeros((1, 1), dtype=np.float32), 2.0)
    walk_case("edge_n2", np.array([[0, 1], [1, 0]], dtype=np.float32), 0.7)

    # The reference test families, exponentiated as 1j*A (drop-in path).
    def expm_case(name, X, with_taylor=True):
        entry = {"X": X, "U_scipy": sl.expm(X)}
        if X.dtype == np.complex64:
            entry["U_scipy_f64"] = sl.expm(X.astype(np.complex128))
        if with_taylor:
            entry["U_taylor"] = taylor(X.astype(np.complex128), m=100)
        cases[name] = entry
        meta[name] = {"kind": "expm", "n": X.shape[0], "dtype": str(X.dtype)}

    for n in (16, 33):
        expm_case(f"complete_n{n}_c64", (1j * graphs.complete(n)).astype(np.complex64))
        expm_case(f"complete_n{n}_c128", (1j * graphs.complete(n, np.float64)).astype(np.complex128))
    expm_case("gnp005_n64_c64", (1j * graphs.erdos_renyi(64, 0.05, seed=41)).astype(np.complex64))
    expm_case("reg4_n32_c128", (1j * graphs.random_regular(32, 4, seed=42, dtype=np.float64)))
    rng = np.random.default_rng(0)
    for n, dt in ((24, np.complex64), (40, np.complex128)):
        ar = graphs.erdos_renyi(n, 0.05, seed=43).astype(np.float64)
        X = (ar + 1j * rng.random((n, n))).astype(dt)
        expm_case(f"perf_general_n{n}_{np.dtype(dt).name}", X, with_taylor=False)
    expm_case("zero_n4_c64", np.zeros((4, 4), dtype=np.complex64), with_taylor=False)

    out = os.path.join(HERE, "golden_cases.npz")
    flat = {}
    for name, entry in cases.items():
        for k, v in entry.items():
            flat[f"{name}::{k}"] = np.asarray(v)
    np.savez_compressed(out, **flat)
    with open(os.path.join(HERE, "golden_cases.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "Crinton/FastCTQW CPU path (scipy.linalg.expm)",
                   "scipy": sl.__dict__.get("__version__", None) or __import__("scipy").__version__,
                   "numpy": np.__version__, "cases": meta}, f, indent=1)
    print("wrote", out, os.path.getsize(out), "bytes,", len(cases), "cases")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FASTCTQW_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set FASTCTQW_REFERENCE_ROOT)")
    main(root)
