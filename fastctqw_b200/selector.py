"""Learned (m, s) selection for the walk exponential: features, training data, training, weights.

The Al-Mohy & Higham selection (the reference's ``scipy.linalg.expm``, FastCTQW/Operator.py:76)
picks the scaling s so that the Pade truncation error stays below the double-precision unit
roundoff 2^-53, from 1-norm bounds of the powers of the generator.  A walk needs much less: an
infidelity of 1e-10, or a relative error of 1e-6 in U.  For walk generators X = -iHt with a real
symmetric H (after the exact trace and rank-one shifts, Y = iB with B real symmetric) the
truncation error has a closed form: the [m/m] Pade approximant maps the imaginary axis onto the
unit circle, so at an eigenvalue i lambda it only rotates the phase, by

    phi_m(x) = 2 arg p_m(ix) - x,   x = lambda / 2^s,   and after s squarings 2^s phi_m(x).

With rho_up = min(||Y||_1, ||Y^4||_1^(1/4), ||Y^6||_1^(1/6)) >= spectral radius (exact norms
of the powers the pipeline forms anyway), the engine *certifies* a choice (m, s) when
2^s |phi_m(rho_up / 2^s)| <= 1e-6 (``certified``; the same test runs in C++ in fx_batch.cu).

The engine also estimates the spectral radius by Lanczos (30 steps from two pseudo-random
starts, ``rho_L``; Ritz values lie inside the spectrum, so rho_L <= rho).  On dense graphs the
norm bound rho_up is about 1.5 rho, which costs a squaring or two.

The learned selector is an MLP 8 -> 64 -> 64 -> (5 logits over m in {3, 5, 7, 9, 13} + s) with
hand-written CUDA kernels (fx_selector.cu: BF16 inference, fused FP32 forward/backward, Adam).
It is trained on the GPU on labels *measured* by the engine (``make_dataset_measured``): every
training walk runs at a grid of forced (m, s) and its result is compared with the FP64
eigendecomposition on the state that exposes the truncation error most, the equal superposition
of the eigenvectors at the two ends of the spectrum; the label is the cheapest (m, s) whose
infidelity stays <= 1e-10.  At run time a proposal is used only when it is cheaper than the
estimated choice (the phase bound at min(rho_up, 1.1 rho_L), at 1e-6), that bound at the proposal
stays below 1e-5 (``gate``) and the result passes the a-posteriori checks; otherwise the
estimated choice (or the plain one, when that is cheaper) is used.

Features (per walk): log2 n, log2 ||Y||_1, log2 (||X||_F / sqrt n), log2 (1 + max off-diagonal
nonzeros of a row), log2 rho_L, rank-one shift flag, log2 d4, log2 d6.
"""
from __future__ import annotations

import hashlib
import json
import ctypes
import math
import os

import numpy as np

from . import _native
from ._native import lib

DEGREES = (3, 5, 7, 9, 13)
PRODUCTS = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}
PHASE_TOL = 1e-6
GATE_TOL = 1e-5      # phase error of the learned selection's gate: infidelity <= 1e-10 for any state
LAN_MARGIN = 0.10    # relative margin on the Lanczos estimate
INFID_LABEL = 1e-10  # measured labels: the cheapest (m, s) at or below this infidelity
X_LIMIT = {3: 5.0, 5: 7.2, 7: 9.3, 9: 11.4, 13: 15.6}   # half of where |phi_m| reaches pi
N_PARAMS = 5126
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "selector_weights.npz")
FEATURE_NAMES = ("log2 n", "log2 ||Y||_1", "log2 ||X||_F/sqrt(n)", "log2(1+max degree)",
                 "log2 rho_L", "rank-one shift", "log2 d4", "log2 d6")


def pade_coeffs(m: int) -> list[float]:
    f = math.factorial
    return [f(2 * m - j) / (f(j) * f(m - j)) for j in range(m + 1)]


def phase_error(m: int, x) -> np.ndarray:
    """phi_m(x) = 2 arg p_m(ix) - x wrapped to (-pi, pi]: the rotation of e^{ix} by r_m."""
    b = pade_coeffs(m)
    x = np.asarray(x, dtype=np.float64)
    z = 1j * x
    acc = np.zeros_like(z)
    for j in range(m, -1, -1):
        acc = acc * z + b[j]
    return np.remainder(2.0 * np.arctan2(acc.imag, acc.real) - x + np.pi, 2 * np.pi) - np.pi


def certified(m: int, s: int, rho_up: float, tol: float = PHASE_TOL) -> bool:
    x = math.ldexp(rho_up, -s)
    return x <= X_LIMIT[m] and math.ldexp(abs(float(phase_error(m, x))), s) <= tol


def certified_choice(rho_up: float, tol: float = PHASE_TOL) -> tuple[int, int]:
    """Cheapest (m, s) (products pi_m + s, ties to the larger m) that the bound certifies."""
    best = None
    for m in DEGREES:
        s = 0
        while s < 200 and not certified(m, s, rho_up, tol):
            s += 1
        cost = PRODUCTS[m] + s
        if best is None or cost <= best[0]:
            best = (cost, m, s)
    return best[1], best[2]


# ------------------------------------------------------------------------------- data
def make_walks(count: int, seed: int, nmin: int = 64, nmax: int = 1024, tmin: float = 0.1,
               tmax: float = 1000.0):
    """Seeded walk generators X = -1j H t: random d-regular (d 3..16), G(n, p) (p 0.05..0.5) or
    uniform-[0, 1]-weighted complete graphs, H = -A or -(D - A), t log-uniform; yields (X, meta)."""
    from . import graphs
    rng = np.random.default_rng(seed)
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        kind = ("regular", "er", "weighted")[int(rng.integers(0, 3))]
        lap = bool(rng.integers(0, 2))
        t = float(math.exp(rng.uniform(math.log(tmin), math.log(tmax))))
        gseed = int(rng.integers(0, 2 ** 31 - 1))
        if kind == "regular":
            d = int(rng.integers(3, 17))
            if (n * d) % 2:
                d += 1
            A = graphs.random_regular(n, d, gseed, np.float64)
        elif kind == "er":
            A = graphs.erdos_renyi(n, float(rng.uniform(0.05, 0.5)), gseed, np.float64)
        else:
            A = graphs.weighted_complete(n, gseed, np.float64)
        H = -((np.diag(A.sum(axis=1)) - A) if lap else A)
        yield np.asarray(-1j * H * t, dtype=np.complex64), (kind, n, lap, t)


def make_dataset(count: int, seed: int, nmin: int = 64, nmax: int = 1024, tmin: float = 0.1,
                 tmax: float = 1000.0, chunk: int = 192) -> dict:
    """The walks of ``make_walks`` run through the engine's analyze-only mode (GPU): features,
    the Al-Mohy & Higham (m, s) and the certified (m, s), the training label."""
    from .batch import WalkBatch
    feats, pm, ps, cm, cs, meta = [], [], [], [], [], []
    it = make_walks(count, seed, nmin, nmax, tmin, tmax)
    todo = count
    while todo > 0:
        k = min(chunk, todo)
        Xs = []
        for _ in range(k):
            X, mt = next(it)
            Xs.append(X)
            meta.append(mt)
        b = WalkBatch([X.shape[0] for X in Xs], analyze_only=True)
        b.run(Xs)
        d = b.details()
        b.close()
        feats.append(d["features"])
        pm.append(d["plain_m"])
        ps.append(d["plain_s"])
        cm.append(d["cert_m"])
        cs.append(d["cert_s"])
        todo -= k
    cat = np.concatenate
    return {"features": cat(feats).astype(np.float32), "plain_m": cat(pm), "plain_s": cat(ps),
            "cert_m": cat(cm), "cert_s": cat(cs), "meta": np.array(meta, dtype=object)}


def min_certified_s(m: int, rho: float, tol: float = PHASE_TOL) -> int:
    s = 0
    while s < 60 and not certified(m, s, rho, tol):
        s += 1
    return s


CHUNK_KEYS = ("features", "plain_m", "plain_s", "cert_m", "cert_s", "label_m", "label_s", "infidelity_plain")


def chunk_cache_path(cache_dir: str, index: int, **args) -> str:
    """File of one chunk of a measured sweep, keyed by every argument that shapes it (the walks
    come from a seeded generator, so the same arguments give the same chunk)."""
    key = json.dumps(args, sort_keys=True)
    h = hashlib.sha1(key.encode()).hexdigest()[:16]
    return os.path.join(cache_dir, f"labels_{h}_chunk{index:04d}.npz")


def save_chunk(path: str, arrays: dict, meta: list) -> None:
    """Write a chunk atomically (a sweep killed while writing leaves no partial file)."""
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".part.npz"
    np.savez(tmp, meta=np.array(json.dumps(meta)), **{k: arrays[k] for k in CHUNK_KEYS})
    os.replace(tmp, path)


def load_chunk(path: str) -> tuple[dict, list]:
    with np.load(path, allow_pickle=False) as z:
        arrays = {k: np.array(z[k]) for k in CHUNK_KEYS}
        meta = [tuple(m) for m in json.loads(str(z["meta"]))]   # (kind, n, laplacian, t) per walk
    return arrays, meta


def make_dataset_measured(count: int, seed: int, nmin: int = 64, nmax: int = 2048, tmin: float = 0.1,
                          tmax: float = 1000.0, chunk: int = 96, depth: int = 5, form: str = "plain",
                          cache_dir: str | None = None) -> dict:
    """Walks of ``make_walks`` with labels measured on the GPU.

    Per chunk of walks: one analyze-only run (features, the Al-Mohy & Higham and the certified
    (m, s)); the FP64 eigendecomposition of every B = Im X (torch on the device) gives the test
    state psi0 = (v_max + v_min) / sqrt 2, whose output is the most sensitive one to phase errors
    (the two ends of the spectrum rotate in opposite directions); then for every m the walks run
    at forced s = s_m - k, k = 0 .. depth - 1, where s_m is the smallest s the rigorous bound
    certifies for that m.  (m, s) passes when the infidelity against the FP64 state is <= 1e-10
    (and no a-posteriori check redid the walk); the label is the cheapest (m, s) (products
    pi_m + s, ties to the larger m) whose s and every larger tested s pass.  The sweeps run in the
    given precision form (the one the selection will serve).

    With ``cache_dir``, every finished chunk is written there (``chunk_cache_path``) and a chunk
    found there is read back instead of measured again, so that an interrupted sweep resumes
    where it stopped."""
    feats, pm_, ps_, cm_, cs_, lm_, ls_, meta, inf_plain = [], [], [], [], [], [], [], [], []
    key_args = dict(count=count, seed=seed, nmin=nmin, nmax=nmax, tmin=tmin, tmax=tmax, chunk=chunk,
                    depth=depth, form=form)
    it = make_walks(count, seed, nmin, nmax, tmin, tmax)
    todo = count
    index = -1
    while todo > 0:
        k = min(chunk, todo)
        todo -= k
        index += 1
        Xs, ms = [], []
        for _ in range(k):
            X, mt = next(it)
            Xs.append(X)
            ms.append(mt)
        path = chunk_cache_path(cache_dir, index, **key_args) if cache_dir else None
        if path and os.path.exists(path):
            arrays, mt = load_chunk(path)
            for lst, key in ((feats, "features"), (pm_, "plain_m"), (ps_, "plain_s"), (cm_, "cert_m"),
                             (cs_, "cert_s"), (lm_, "label_m"), (ls_, "label_s"), (inf_plain, "infidelity_plain")):
                lst.append(arrays[key])
            meta.extend(mt)
            continue
        res = _measure_chunk(Xs, depth, form)
        for lst, key in ((feats, "features"), (pm_, "plain_m"), (ps_, "plain_s"), (cm_, "cert_m"),
                         (cs_, "cert_s"), (lm_, "label_m"), (ls_, "label_s"), (inf_plain, "infidelity_plain")):
            lst.append(res[key])
        meta.extend(ms)
        if path:
            save_chunk(path, res, ms)
    cat = np.concatenate
    return {"features": cat(feats).astype(np.float32), "plain_m": cat(pm_), "plain_s": cat(ps_),
            "cert_m": cat(cm_), "cert_s": cat(cs_), "label_m": cat(lm_), "label_s": cat(ls_),
            "infidelity_plain": cat(inf_plain), "meta": np.array(meta, dtype=object)}


def _measure_chunk(Xs: list, depth: int, form: str) -> dict:
    """Labels of one chunk of walks by forced sweeps on the GPU (make_dataset_measured)."""
    import torch
    from .batch import OPT_SAMPLE_WALKS, WalkBatch
    dev = torch.device("cuda", 0)
    k = len(Xs)
    ns = [X.shape[0] for X in Xs]
    with WalkBatch(ns, analyze_only=True) as b:
        b.run(Xs)
        d = b.details()
    ru = rho_up(d["features"])
    dX = [torch.from_numpy(X).to(dev) for X in Xs]
    p0s, refs = [], []
    for X in Xs:
        lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to(dev))
        p = (V[:, -1] + V[:, 0]) / math.sqrt(2.0)
        ref = (torch.exp(1j * lam[-1]) * V[:, -1] + torch.exp(1j * lam[0]) * V[:, 0]) / math.sqrt(2.0)
        p0s.append(p.to(torch.complex64))
        refs.append(ref)
        del lam, V
    outs = [torch.empty_like(p) for p in p0s]
    sweep = WalkBatch(ns, form=form)
    sweep.set_option(OPT_SAMPLE_WALKS, 0)

    def infidelities():
        sweep.run_device(dX, p0s, outs)
        torch.cuda.synchronize()
        oc = sweep.details()["outcome"]
        r = []
        for w in range(k):
            q = outs[w].to(torch.complex128)
            ov = torch.vdot(refs[w], q).abs() ** 2 / (torch.vdot(q, q).real * torch.vdot(refs[w], refs[w]).real)
            r.append(1.0 if oc[w] == -2 else float(1.0 - ov))
        return np.array(r)

    inf_plain = infidelities()   # the plain selection's own result
    best = [(PRODUCTS[int(d["plain_m"][w])] + int(d["plain_s"][w]), int(d["plain_m"][w]), int(d["plain_s"][w]))
            for w in range(k)]
    for m in DEGREES:
        s_top = np.array([min_certified_s(m, float(r)) for r in ru])
        ok = np.ones(k, dtype=bool)     # every s tested so far (from the top) passed
        for kk in range(depth):
            s_try = s_top - kk
            active = ok & (s_try >= 0)
            if not active.any():
                break
            sweep.force_selection(np.full(k, m), np.maximum(s_try, 0))
            inf = infidelities()
            for w in np.nonzero(active)[0]:
                if inf[w] <= INFID_LABEL:
                    cost = PRODUCTS[m] + int(s_try[w])
                    if cost < best[w][0] or (cost == best[w][0] and m > best[w][1]):
                        best[w] = (cost, m, int(s_try[w]))
                else:
                    ok[w] = False
    sweep.force_selection()
    sweep.close()
    res = {"features": np.asarray(d["features"], dtype=np.float32), "plain_m": d["plain_m"],
           "plain_s": d["plain_s"], "cert_m": d["cert_m"], "cert_s": d["cert_s"],
           "label_m": np.array([b_[1] for b_ in best], dtype=np.int32),
           "label_s": np.array([b_[2] for b_ in best], dtype=np.int32),
           "infidelity_plain": inf_plain}
    del dX, p0s, refs, outs
    torch.cuda.empty_cache()
    return res


def merge(*sets: dict) -> dict:
    return {k: np.concatenate([d[k] for d in sets]) for k in sets[0]}


def rho_up(features: np.ndarray) -> np.ndarray:
    """min(||Y||_1, d4, d6) from the features (columns 1, 6, 7 are their log2)."""
    f = np.asarray(features, dtype=np.float64)
    return np.exp2(np.minimum(f[:, 1], np.minimum(f[:, 6], f[:, 7])))


def rho_gate(features: np.ndarray) -> np.ndarray:
    """min(rho_up, 1.1 rho_L): the spectral radius as far as the engine knows it."""
    f = np.asarray(features, dtype=np.float64)
    return np.minimum(rho_up(f), np.exp2(f[:, 4]) * (1.0 + LAN_MARGIN))


def gate(features, plain_m, plain_s, prop_m, prop_s) -> np.ndarray:
    """Selection outcome per walk, as the engine decides it: 2 proposal accepted, 3 estimated
    choice (the proposal rejected by the bound or not cheaper), -1 rejected with the plain
    choice kept, 0 plain choice (nothing cheaper)."""
    r = rho_gate(features)
    em, es = estimated_choice(features)
    out = np.zeros(len(r), dtype=np.int32)
    for i in range(len(r)):
        cost = PRODUCTS[int(plain_m[i])] + int(plain_s[i])
        if PRODUCTS[int(em[i])] + int(es[i]) < cost:
            out[i] = 3
            cost = PRODUCTS[int(em[i])] + int(es[i])
        pm, ps = int(prop_m[i]), int(prop_s[i])
        if PRODUCTS[pm] + ps < cost:
            if certified(pm, ps, float(r[i]), GATE_TOL):
                out[i] = 2
            elif out[i] != 3:
                out[i] = -1
    return out


def estimated_choice(features) -> tuple[np.ndarray, np.ndarray]:
    """The engine's estimated selection (selector 3) for every walk: the cheapest (m, s) the
    phase bound at min(rho_up, 1.1 rho_L) certifies at 1e-6."""
    r = rho_gate(features)
    mm, ss = zip(*[certified_choice(float(x)) for x in r])
    return np.array(mm, dtype=np.int32), np.array(ss, dtype=np.int32)


def labels(ds: dict) -> tuple[np.ndarray, np.ndarray]:
    """Class index of the label m in DEGREES and the label s (float): the measured labels when
    the dataset has them, else the certified choice."""
    km, ks = ("label_m", "label_s") if "label_m" in ds else ("cert_m", "cert_s")
    idx = {m: i for i, m in enumerate(DEGREES)}
    return (np.array([idx[int(m)] for m in ds[km]], dtype=np.int32), np.asarray(ds[ks], dtype=np.float32))


# ----------------------------------------------------------------------------- network
def init_weights(seed: int) -> np.ndarray:
    """He-initialised FP32 weights in the kernel's layout (W1, b1, W2, b2, W3, b3)."""
    rng = np.random.default_rng(seed)
    w1 = rng.standard_normal((64, 8)) * math.sqrt(2 / 8)
    w2 = rng.standard_normal((64, 64)) * math.sqrt(2 / 64)
    w3 = rng.standard_normal((6, 64)) * math.sqrt(1 / 64)
    return np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3.ravel(),
                           np.zeros(6)]).astype(np.float32)


def fold_standardisation(w: np.ndarray, mean: np.ndarray, std: np.ndarray) -> np.ndarray:
    """Weights that take raw features: W1 x' + b1 with x' = (x - mean) / std."""
    w = w.copy()
    W1 = w[:512].reshape(64, 8) / std[None, :]
    w[512:576] = w[512:576] - W1 @ mean
    w[:512] = W1.ravel()
    return w


def _dev(a, dtype):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def train(ds: dict, epochs: int = 60, batch: int = 256, lr: float = 2e-3, lam: float = 0.25,
          seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Train on the GPU (fx_mlp_train).  Returns (weights for raw features, loss per epoch)."""
    import torch
    X = np.asarray(ds["features"], dtype=np.float32)
    mean, std = X.mean(axis=0), X.std(axis=0) + 1e-6
    ym, ys = labels(ds)
    w = _dev(init_weights(seed), torch.float32)
    dx = _dev((X - mean) / std, torch.float32)
    dym, dys = _dev(ym, torch.int32), _dev(ys, torch.float32)
    losses = (ctypes.c_float * epochs)()
    rc = lib().fx_mlp_train(w.data_ptr(), dx.data_ptr(), dym.data_ptr(), dys.data_ptr(), len(X), epochs,
                            batch, lr, lam, seed, losses, torch.cuda.current_stream().cuda_stream)
    if rc != _native.OK:
        raise RuntimeError(lib().fx_mlp_error().decode())
    return fold_standardisation(w.cpu().numpy(), mean, std), np.array(losses[:], dtype=np.float32)


def infer(w: np.ndarray, features: np.ndarray) -> np.ndarray:
    """n x 6 outputs of the network (BF16 inference kernel)."""
    import torch
    dw = _dev(w, torch.float32)
    dx = _dev(np.asarray(features, dtype=np.float32), torch.float32)
    out = torch.empty((len(features), 6), dtype=torch.float32, device="cuda")
    rc = lib().fx_mlp_infer(dw.data_ptr(), dx.data_ptr(), len(features), out.data_ptr(),
                            torch.cuda.current_stream().cuda_stream)
    if rc != _native.OK:
        raise RuntimeError(lib().fx_mlp_error().decode())
    torch.cuda.synchronize()
    return out.cpu().numpy()


def proposals(out: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(m, s) proposed by network outputs (argmax of the logits, s rounded, >= 0)."""
    m = np.array([DEGREES[int(i)] for i in np.argmax(out[:, :5], axis=1)], dtype=np.int32)
    s = np.maximum(0, np.rint(out[:, 5])).astype(np.int32)
    return m, s


# ----------------------------------------------------------------------------- weights
def save(path: str, w: np.ndarray, **meta) -> None:
    np.savez(path, weights=np.asarray(w, dtype=np.float32), **meta)


def load(path: str = WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        w = np.asarray(z["weights"], dtype=np.float32)
    if w.size != N_PARAMS:
        raise ValueError(f"selector weights: expected {N_PARAMS} values, found {w.size}")
    return w


def set_weights(w: np.ndarray | None = None) -> None:
    """Install weights for the learned selection of every handle (default: the shipped file)."""
    w = np.ascontiguousarray(load() if w is None else w, dtype=np.float32)
    rc = lib().fx_selector_set_weights(w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), w.size)
    if rc != _native.OK:
        raise RuntimeError(lib().fx_batch_last_error(None).decode())
