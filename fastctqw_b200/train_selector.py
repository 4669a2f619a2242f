"""Train the learned (m, s) selector on the GPU from measured labels and write its weights and
an evaluation report.

    python -m fastctqw_b200.train_selector [--train 2048] [--test 512] [--epochs 120] [--cache-dir DIR]

1. training and held-out sets from seeded walk generators (selector.make_walks), labelled by
   measured sweeps (selector.make_dataset_measured): every walk runs at a grid of forced (m, s),
   its state is compared with the FP64 eigendecomposition on the most phase-sensitive state,
   and the label is the cheapest (m, s) at infidelity <= 1e-10;
2. training with the project's kernels (fx_mlp_train: fused forward/backward + Adam);
3. held-out evaluation: label accuracy, acceptance of the gate, and the products (Pade products
   + squarings) per walk of the plain (Al-Mohy & Higham), certified, estimated (Lanczos), learned
   and measured-best selections;
4. end to end on held-out walks: each selector run through the batch engine, infidelity against
   the FP64 state and the squarings taken.
Writes fastctqw_b200/data/selector_weights.npz and fastctqw_b200/data/selector_eval.json.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import selector

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


def products(m, s) -> np.ndarray:
    return np.array([selector.PRODUCTS[int(a)] + int(b) for a, b in zip(m, s)], dtype=np.float64)


def evaluate(w, ds) -> dict:
    out = selector.infer(w, ds["features"])
    pm, ps = selector.proposals(out)
    ym, ys = selector.labels(ds)
    outcome = selector.gate(ds["features"], ds["plain_m"], ds["plain_s"], pm, ps)
    plain = products(ds["plain_m"], ds["plain_s"])
    cert = np.minimum(plain, products(ds["cert_m"], ds["cert_s"]))
    em, es = selector.estimated_choice(ds["features"])
    est = np.minimum(plain, products(em, es))
    label = products(ds["label_m"], ds["label_s"])
    learned = np.where(outcome == 2, products(pm, ps), np.where(outcome == 3, est, plain))
    return {
        "instances": int(len(plain)),
        "label_m_accuracy": float(np.mean(pm == ds["label_m"])),
        "label_s_accuracy": float(np.mean(ps == ds["label_s"])),
        "label_s_mae": float(np.mean(np.abs(out[:, 5] - ys))),
        "accepted": int((outcome == 2).sum()),
        "estimated_fallback": int((outcome == 3).sum()),
        "rejected_plain_kept": int((outcome == -1).sum()),
        "below_measured_label": int(np.sum((outcome == 2) & (products(pm, ps) < label))),
        "products_per_walk": {"plain": float(plain.mean()), "certified": float(cert.mean()),
                              "estimated": float(est.mean()), "learned": float(learned.mean()),
                              "measured_best": float(label.mean())},
    }


def end_to_end(w, count: int, seed: int, nmin: int, nmax: int, form: str = "plain") -> dict:
    """Every selector on fresh walks through the batch engine; infidelity against the FP64 state
    of psi0 = (v_max + v_min) / sqrt 2 (the most phase-sensitive state) and squarings taken."""
    import torch
    from .batch import WalkBatch
    dev = torch.device("cuda", 0)
    walks = list(selector.make_walks(count, seed, nmin, nmax, 0.1, 1000.0))
    Xs = [X for X, _ in walks]
    ns = [X.shape[0] for X in Xs]
    dX = [torch.from_numpy(X).to(dev) for X in Xs]
    p0s, refs = [], []
    for X in Xs:
        lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to(dev))
        p0s.append(((V[:, -1] + V[:, 0]) / math.sqrt(2.0)).to(torch.complex64))
        refs.append((torch.exp(1j * lam[-1]) * V[:, -1] + torch.exp(1j * lam[0]) * V[:, 0]) / math.sqrt(2.0))
    selector.set_weights(w)
    res = {"walks": count, "n_range": [nmin, nmax]}
    for mode in ("plain", "certified", "estimated", "learned"):
        outs = [torch.empty_like(p) for p in p0s]
        with WalkBatch(ns, selector=mode, form=form) as b:
            b.run_device(dX, p0s, outs)
            torch.cuda.synchronize()
            m, s = b.selection()
            oc = b.details()["outcome"]
        inf = []
        for k in range(count):
            q = outs[k].to(torch.complex128)
            ov = torch.vdot(refs[k], q).abs() ** 2 / (torch.vdot(q, q).real * torch.vdot(refs[k], refs[k]).real)
            inf.append(float(1.0 - ov))
        res[mode] = {"max_infidelity": max(inf), "squarings": int(s.sum()),
                     "products": float(products(m, s).sum()),
                     "outcomes": {int(a): int(c) for a, c in zip(*np.unique(oc, return_counts=True))}}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2048)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--nmax", type=int, default=2048)
    ap.add_argument("--train-large", type=int, default=128, help="extra training walks with n in [nmax, nmax-large]")
    ap.add_argument("--test-large", type=int, default=32)
    ap.add_argument("--nmax-large", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=120)
    ap.add_argument("--e2e", type=int, default=192)
    ap.add_argument("--form", default="mixed", choices=["plain", "mixed"],
                    help="precision form of the measured sweeps (the form the selection serves)")
    ap.add_argument("--out", default=os.path.join(DATA, "selector_weights.npz"))
    ap.add_argument("--report", default=os.path.join(DATA, "selector_eval.json"))
    ap.add_argument("--cache-dir", default=None,
                    help="keep every measured chunk of labels here and read back the ones found, so that an "
                         "interrupted sweep resumes where it stopped")
    a = ap.parse_args(argv)
    t0 = time.time()
    c = a.cache_dir
    ds_train = selector.merge(selector.make_dataset_measured(a.train, seed=1, nmax=a.nmax, form=a.form, cache_dir=c),
                              selector.make_dataset_measured(a.train_large, seed=4, nmin=a.nmax,
                                                             nmax=a.nmax_large, chunk=16, form=a.form, cache_dir=c))
    ds_test = selector.merge(selector.make_dataset_measured(a.test, seed=2, nmax=a.nmax, form=a.form, cache_dir=c),
                             selector.make_dataset_measured(a.test_large, seed=5, nmin=a.nmax,
                                                            nmax=a.nmax_large, chunk=16, form=a.form, cache_dir=c))
    t1 = time.time()
    w, losses = selector.train(ds_train, epochs=a.epochs)
    t2 = time.time()
    selector.save(a.out, w, losses=losses)
    rep = {"form": a.form, "labels": "measured: cheapest (m, s) with infidelity <= 1e-10 against the FP64 state of "
                     "(v_max + v_min)/sqrt(2), over forced sweeps s = s_cert(m) - k, k < 5, m in {3,5,7,9,13}",
           "train": a.train + a.train_large, "test": a.test + a.test_large, "n_range": [64, a.nmax_large],
           "t_range": [0.1, 1000.0], "epochs": a.epochs,
           "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
           "seconds_labels": round(t1 - t0, 1), "seconds_train": round(t2 - t1, 1),
           "plain_selection_max_infidelity_train": float(np.max(ds_train["infidelity_plain"])),
           "train_eval": evaluate(w, ds_train), "heldout": evaluate(w, ds_test)}
    rep["end_to_end"] = end_to_end(w, a.e2e, seed=3, nmin=64, nmax=a.nmax, form=a.form)
    with open(a.report, "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
