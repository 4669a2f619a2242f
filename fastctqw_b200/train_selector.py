"""Train the learned (m, s) selector on the GPU and write its weights and an evaluation report.

    python -m fastctqw_b200.train_selector [--train 8000] [--test 2000] [--epochs 80]

1. training and held-out sets from seeded walk generators (selector.make_walks), labelled by the
   engine's analyze-only runs (the cheapest (m, s) the truncation bound certifies);
2. training with the project's kernels (fx_mlp_train: fused forward/backward + Adam);
3. held-out evaluation: label accuracy, acceptance / fallback rate of the gate, products saved
   against the Al-Mohy & Higham choice (and against the certified choice, the ceiling);
4. end-to-end walks with the learned selection on a held-out subset, infidelity against the
   FP64 eigendecomposition of H and against the plain selection's result.
Writes fastctqw_b200/data/selector_weights.npz and fastctqw_b200/data/selector_eval.json.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import selector

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def evaluate(w, ds) -> dict:
    out = selector.infer(w, ds["features"])
    pm, ps = selector.proposals(out)
    ym, ys = selector.labels(ds)
    outcome = selector.gate(ds["features"], ds["plain_m"], ds["plain_s"], pm, ps)
    P = selector.PRODUCTS
    plain = np.array([P[int(m)] + int(s) for m, s in zip(ds["plain_m"], ds["plain_s"])])
    cert = np.array([P[int(m)] + int(s) for m, s in zip(ds["cert_m"], ds["cert_s"])])
    chosen = np.where(outcome == 2, np.array([P[int(m)] + int(s) for m, s in zip(pm, ps)]), plain)
    cheaper = outcome != 0
    return {
        "instances": int(len(plain)),
        "label_m_accuracy": float(np.mean(pm == ds["cert_m"])),
        "label_s_accuracy": float(np.mean(ps == ds["cert_s"])),
        "label_s_mae": float(np.mean(np.abs(out[:, 5] - ys))),
        "proposals_cheaper_than_plain": int(cheaper.sum()),
        "accepted": int((outcome == 2).sum()),
        "fallback_rate": float(np.mean(outcome[cheaper] == -1)) if cheaper.any() else 0.0,
        "products_plain_mean": float(plain.mean()),
        "products_learned_mean": float(chosen.mean()),
        "products_certified_mean": float(cert.mean()),
        "products_saved_per_walk": float((plain - chosen).mean()),
        "squarings_saved_per_walk": float(np.mean(np.where(outcome == 2, ds["plain_s"] - ps, 0))),
    }


def end_to_end(w, count: int, seed: int) -> dict:
    """Learned vs plain selection on fresh walks (n <= 384), both against FP64 eigh."""
    from .batch import WalkBatch
    walks = list(selector.make_walks(count, seed, 48, 384, 0.1, 200.0))
    Xs = [X for X, _ in walks]
    psi0 = [np.full(X.shape[0], 1 / np.sqrt(X.shape[0]), np.complex64) for X in Xs]
    psi0 = [p if k % 2 else np.eye(X.shape[0], dtype=np.complex64)[k % X.shape[0]] for k, (p, X) in
            enumerate(zip(psi0, Xs))]
    res = {}
    selector.set_weights(w)
    for mode in ("plain", "learned"):
        b = WalkBatch([X.shape[0] for X in Xs], selector=mode)
        res[mode] = (b.run(Xs, psi0), b.selection(), b.details())
        b.close()
    inf_l, inf_p, sq_l, sq_p = [], [], 0, 0
    for k, X in enumerate(Xs):
        B = (X.astype(np.complex128) / 1j).real
        lam, V = np.linalg.eigh(B)
        ref = V @ (np.exp(1j * lam) * (V.T @ psi0[k].astype(np.complex128)))
        for mode, acc in (("learned", inf_l), ("plain", inf_p)):
            psi = res[mode][0][k].astype(np.complex128)
            acc.append(1 - abs(np.vdot(ref, psi)) ** 2 / (np.vdot(psi, psi).real * np.vdot(ref, ref).real))
        sq_l += int(res["learned"][1][1][k])
        sq_p += int(res["plain"][1][1][k])
    oc = res["learned"][2]["outcome"]
    return {"walks": count, "max_infidelity_learned": float(max(inf_l)), "max_infidelity_plain": float(max(inf_p)),
            "squarings_learned": sq_l, "squarings_plain": sq_p,
            "accepted": int((oc == 2).sum()), "rejected_by_bound": int((oc == -1).sum()),
            "rejected_by_unitarity": int((oc == -2).sum())}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=8000)
    ap.add_argument("--test", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=80)
    ap.add_argument("--nmax", type=int, default=1024)
    ap.add_argument("--train-large", type=int, default=1200, help="extra training walks with n in [nmax, nmax-large]")
    ap.add_argument("--test-large", type=int, default=300)
    ap.add_argument("--nmax-large", type=int, default=4096)
    ap.add_argument("--e2e", type=int, default=64)
    ap.add_argument("--out", default=os.path.join(DATA, "selector_weights.npz"))
    ap.add_argument("--report", default=os.path.join(DATA, "selector_eval.json"))
    a = ap.parse_args(argv)
    t0 = time.time()
    ds_train = selector.merge(selector.make_dataset(a.train, seed=1, nmax=a.nmax),
                              selector.make_dataset(a.train_large, seed=4, nmin=a.nmax, nmax=a.nmax_large,
                                                    chunk=32))
    ds_test = selector.merge(selector.make_dataset(a.test, seed=2, nmax=a.nmax),
                             selector.make_dataset(a.test_large, seed=5, nmin=a.nmax, nmax=a.nmax_large,
                                                   chunk=32))
    t1 = time.time()
    w, losses = selector.train(ds_train, epochs=a.epochs)
    t2 = time.time()
    selector.save(a.out, w, losses=losses)
    rep = {"train": a.train + a.train_large, "test": a.test + a.test_large, "n_range": [64, a.nmax_large],
           "t_range": [0.1, 1000.0],
           "epochs": a.epochs, "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
           "seconds_data": round(t1 - t0, 1), "seconds_train": round(t2 - t1, 1),
           "train_eval": evaluate(w, ds_train), "heldout": evaluate(w, ds_test)}
    rep["end_to_end"] = end_to_end(w, a.e2e, seed=3)
    with open(a.report, "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
