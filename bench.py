"""Benchmark of the expm(-iHt) walk on B200.

Workload (the dense single-walk configuration): Erdos-Renyi G(n=10000, p=0.5) from a fixed
seed, H = Laplacian D - A (integer entries), t = 4.5, X = -1j*H*t in complex64 (the
reference's Operator convention, FastCTQW/Operator.py:49-56), psi0 = |0>.  One step is one
walk: U = expm(X) by scaling and squaring with Pade, then psi = U psi0, with X resident in
HBM.  Synthetic data generated from the seed (no dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  `value` is ms per walk (lower is better) with inputs in HBM; `e2e`
is the same through the public drop-in API (``ExpMatComplex64.run`` on a host ndarray: the
host->device copy of X and the device->host copy of U are inside the timed region).
With N > 1 (torchrun) each rank runs its own walk (replicas; the single walk does not
shard), and `value` is the job's time divided by the walks of all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "expm(-iHt) ms at N=10k c64; batched walks/s; chosen vs plain @ infid<=1e-10"


def product_traffic_per_launch(form: str):
    """DRAM bytes (read + write) per k_gemm_i8 launch of the benchmark walk in the given form
    ("mixed/chebyshev", "mixed", ...), from the committed summary of an ncu capture of one walk's
    product launches (dram__bytes_read.sum + dram__bytes_write.sum, averaged over the walk's
    launches): the line `dram_bytes_per_launch[<form>]: <bytes>` of
    profiles/k_gemm_i8_walk_traffic.md.  None when the summary has no line for the form."""
    import re
    path = os.path.join(REPO, "profiles", "k_gemm_i8_walk_traffic.md")
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_launch\[" + re.escape(form) + r"\]:\s*([0-9.eE+]+)", text)
    if not m:
        return None
    return {"bytes": float(m.group(1)), "source": "profiles/k_gemm_i8_walk_traffic.md (ncu, one walk's product launches)"}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def workload(n: int, seed: int, t: float):
    from fastctqw_b200 import graphs
    A = graphs.erdos_renyi(n, 0.5, seed=seed, dtype=np.float32)
    L = np.diag(A.sum(axis=1)) - A            # D - A, exact small integers
    H = -1.0 * L                               # Operator._buildHamiltonian(laplacian=True), gamma = 1
    X = np.asarray(-1j * H * t, dtype=np.complex64)   # Operator._buildUnitory
    return A, H.astype(np.float64), X


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i - 5] for r in self.rows for i in range(5, 9) if r[i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_reference_sample(n_sample: int, seed: int, t: float, reps: int):
    """Time the reference's CPU path (scipy.linalg.expm on X, as FastCTQW/Operator.py:76 does)
    on a sample size and return (seconds per call, (m, s) the algorithm picks at that size)."""
    from oracle import expm_oracle as eo
    _, _, Xs = workload(n_sample, seed, t)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        eo.reference_cpu_expm(Xs)
        times.append(time.perf_counter() - t0)
    return min(times), Xs


def scale_to_full(sec_sample: float, Xs: np.ndarray, n_full: int):
    """Extrapolate a CPU time from the sample to the full size with the algorithm's flop count
    8 N^3 (pi_m + s) + (8/3) N^3 + 8 N^3, using (m, s) of each size."""
    from oracle import expm_oracle as eo
    sel_s = eo.select_pade(Xs.astype(np.complex128))
    sel_f = full_size_selection(n_full, Xs.shape[0], (sel_s.m, sel_s.s))
    f_s = eo.flops_expm(Xs.shape[0], sel_s.m, sel_s.s)
    f_f = eo.flops_expm(n_full, sel_f[0], sel_f[1])
    return sec_sample * f_f / f_s, (sel_s.m, sel_s.s), sel_f


def threads_used():
    try:
        from threadpoolctl import threadpool_info
        info = threadpool_info()
        return max((i.get("num_threads", 1) for i in info), default=os.cpu_count())
    except Exception:  # noqa: BLE001
        return os.cpu_count()


def reference_walks(n: int, seed: int, t: float, steps: int, budget_s: float):
    """Full-size runs of the reference's CPU path on this host: X = -1j H t of the benchmark walk,
    U = scipy.linalg.expm(X) (FastCTQW/Operator.py:74-76), psi = U psi0 (FastCTQW/Ctqw.py:94).
    At least one run; more (up to `steps`) only while the runs so far stay within `budget_s`.
    Returns (seconds of every timed run, (m, s) the algorithm picks)."""
    from oracle import expm_oracle as eo
    _, _, X = workload(n, seed, t)
    psi0 = np.zeros(n, dtype=np.complex64)
    psi0[0] = 1.0
    times = []
    while True:
        t0 = time.perf_counter()
        U = eo.reference_cpu_expm(X)
        psi = U @ psi0
        times.append(time.perf_counter() - t0)
        del U, psi
        if len(times) >= max(1, steps) or sum(times) * (len(times) + 1) / len(times) > budget_s:
            break
    sel = eo.select_pade(X.astype(np.complex128)) if n <= 4096 else None
    return times, sel


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (scipy.linalg.expm) on this host's cores, on
    the benchmark's own N.  A full N = 10000 expm takes tens of seconds, so the run times as many
    full walks as fit the step budget (at least one) and reports those steps; no warm-up run (a
    second full run would only double the time)."""
    if rank != 0:
        return
    times, _ = reference_walks(args.n, args.seed, args.t, args.steps, args.ref_budget_s)
    v = 1e3 * statistics.median(times)
    cores = threads_used()
    # labelled cross-check: the earlier flop-model extrapolation from a small sample
    sec, Xs = cpu_reference_sample(args.ref_sample_n, args.seed, args.t, 2)
    model_sec, sel_s, sel_full = scale_to_full(sec, Xs, args.n)
    sample = (f"scipy.linalg.expm + U psi0 (the reference CPU path, FastCTQW/Operator.py:74-76, Ctqw.py:94) "
              f"on the full N={args.n} walk, {len(times)} run(s) timed ({args.steps} requested; runs are "
              f"added only within a {args.ref_budget_s:.0f} s budget), median; OpenBLAS/MKL threads={cores}")
    print(json.dumps({
        "metric": METRIC, "value": round(v, 3), "unit": "ms", "impl": "reference", "n_gpus": world,
        "steps": len(times), "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": round(v, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded G(n,0.5) Laplacian)",
        "config": {"workload": f"dense ER G(n={args.n}, p=0.5) Laplacian, t={args.t}, complex64 expm + U psi0",
                   "n": args.n, "t": args.t},
        "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": cores, "kind": "reference",
                         "sample": sample, "runs_s": [round(x, 2) for x in times]},
        "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "flop_model_cross_check": {"ms": round(model_sec * 1e3, 1),
                                   "from": f"N={args.ref_sample_n} (m={sel_s[0]}, s={sel_s[1]}) scaled to "
                                           f"(m={sel_full[0]}, s={sel_full[1]}) by 8N^3(pi_m+s)+(8/3)N^3+8N^3"},
    }), flush=True)


def full_size_selection(n_full, n_sample, sel_sample):
    """(m, s) of the reference algorithm at the full size.  For this family ||X||_1 and the
    d_p norms grow linearly with N (t * degree ~ t N p), so s grows by log2(N_full/N_sample)
    from the sample's s (scipy picks s = 10, 11, 12 at N = 1024, 2048, 4096 here)."""
    import math
    return (13, sel_sample[1] + int(round(math.log2(n_full / n_sample))))


def accuracy_vs_eigh(H: np.ndarray, t: float, dU, psi_e0, psi_e0_plain, dev, seed: int) -> dict:
    """Accuracy of the timed walk against the FP64 eigendecomposition propagator
    U_ref = V diag(exp(-i lambda t)) V^T of the real symmetric H (torch FP64 on the device):
    the relative Frobenius error of the stored complex64 U, and the infidelity of the states of
    |0> (the walk's own psi), of the uniform superposition and of a seeded random state (psi = U
    psi0 in complex128 from the stored U)."""
    import torch
    from fastctqw_b200 import graphs
    from oracle import expm_oracle as eo
    n = H.shape[0]
    lam, V = torch.linalg.eigh(torch.from_numpy(H).to(dev))
    Vc = V.to(torch.complex128)
    del V
    Uref = (Vc * torch.exp(-1j * lam * t)) @ Vc.T
    del Vc
    torch.cuda.empty_cache()
    out = {"oracle": "FP64 eigendecomposition of H on the device (torch.linalg.eigh)"}
    ref0 = Uref[:, 0].cpu().numpy()
    out["infidelity_e0"] = eo.infidelity(psi_e0.cpu().numpy(), ref0)
    if psi_e0_plain is not None:
        out["infidelity_e0_plain"] = eo.infidelity(psi_e0_plain.cpu().numpy(), ref0)
    U = dU.to(torch.complex128)
    out["u_rel_error"] = float(torch.linalg.matrix_norm(U - Uref) / torch.linalg.matrix_norm(Uref))
    for kind, p0 in (("uniform", graphs.uniform_state(n)), ("random", graphs.random_state(n, seed))):
        p = torch.from_numpy(p0).to(dev).to(torch.complex128)
        out[f"infidelity_{kind}"] = eo.infidelity((U @ p).cpu().numpy(), (Uref @ p).cpu().numpy())
    del U, Uref
    torch.cuda.empty_cache()
    return out


def bench_stress(args, dev) -> dict:
    """The large-norm stress workload: dense symmetric weighted graph, N = 16384, weights uniform
    in [0, 1) from a fixed seed (zero diagonal), H = weighted Laplacian D - W, t = 100, X = -1j H t
    (FastCTQW/Operator.py:49-56).  Runs complex64 in the plain and mixed forms (the mixed form
    with the Pade and with the Chebyshev approximant) and complex128
    (int8 slices on FP64 masters), each timed with CUDA events, with the unitarity residual
    ||U_k^H U_k - I||_F / sqrt(N) after every squaring k (FX_OPT_DRIFT) and the final accuracy
    against the FP64 eigendecomposition of the same generator (the complex64 input is itself a
    rounding of X, so its oracle is the exact propagator of that rounded X)."""
    import torch
    from fastctqw_b200 import graphs
    from fastctqw_b200._native import Engine
    from oracle import expm_oracle as eo
    n, t = args.stress_n, args.stress_t
    Wt = graphs.weighted_complete(n, seed=args.seed, dtype=np.float64)
    L = np.diag(Wt.sum(axis=1)) - Wt
    del Wt
    out = {"workload": f"dense U[0,1)-weighted complete graph N={n}, H = D - W, t={t}",
           "oracle": "FP64 eigendecomposition of the (rounded) generator on the device"}
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for dt, forms in ((np.complex64, (("plain", "pade"), ("mixed", "pade"), ("mixed", "chebyshev"))),
                      (np.complex128, (("plain", "pade"),))):
        X = np.asarray(-1j * (-1.0 * L) * t, dtype=dt)
        lam, V = torch.linalg.eigh(torch.from_numpy(np.ascontiguousarray(X.imag, dtype=np.float64)).to(dev))
        Vc = V.to(torch.complex128)
        del V
        Uref = (Vc * torch.exp(1j * lam)) @ Vc.T
        del Vc, lam
        torch.cuda.empty_cache()
        dX = torch.from_numpy(X).to(dev)
        del X
        p0 = torch.zeros(n, dtype=dX.dtype, device=dev)
        p0[0] = 1.0
        dp = torch.empty_like(p0)
        dU = torch.empty_like(dX)
        eng = Engine(n, dt)
        for form, approx in forms:
            eng.configure(form=form, approx=approx, drift=False)
            eng.walk_device(dX, p0, dp, dU, stream)
            torch.cuda.synchronize()
            ev[0].record(stream)
            eng.walk_device(dX, p0, dp, dU, stream)
            ev[1].record(stream)
            torch.cuda.synchronize()
            st = eng.stats()
            rec = {"ms": round(ev[0].elapsed_time(ev[1]), 2), "m": st["m"], "s": st["s"], "degree": st["degree"]}
            U = dU.to(torch.complex128)
            rec["u_rel_error"] = float(torch.linalg.matrix_norm(U - Uref) / torch.linalg.matrix_norm(Uref))
            rec["infidelity_e0"] = eo.infidelity(dp.cpu().numpy(), Uref[:, 0].cpu().numpy())
            for kind, v in (("uniform", graphs.uniform_state(n)), ("random", graphs.random_state(n, args.seed))):
                pv = torch.from_numpy(v).to(dev).to(torch.complex128)
                rec[f"infidelity_{kind}"] = eo.infidelity((U @ pv).cpu().numpy(), (Uref @ pv).cpu().numpy())
            G = U.conj().T @ U
            G.diagonal().sub_(1.0)
            rec["unitarity_residual_final"] = float(torch.linalg.matrix_norm(G) / np.sqrt(n))
            del U, G
            torch.cuda.empty_cache()
            eng.configure(drift=True)
            eng.walk_device(dX, p0, dp, dU, stream)
            torch.cuda.synchronize()
            rec["drift_per_squaring"] = [float("%.4g" % x) for x in eng.unitarity_drift()]
            eng.configure(drift=False)
            out[f"{np.dtype(dt).name}_{form}" + ("_chebyshev" if approx == "chebyshev" else "")] = rec
        eng.close()
        del dX, dU, Uref
        torch.cuda.empty_cache()
    return out


def batch_workload(count: int, seed: int, nmin: int, nmax: int):
    """The uneven batch: `count` walks, N ~ U{nmin..nmax}, alternating random d-regular
    (d ~ U{3..16}) and G(N, p) (p ~ U[0.05, 0.5]) adjacency graphs, t log-uniform in [0.5, 50],
    X = -1j*H*t with H = -A (FastCTQW/Operator.py:49-56) in complex64, psi0 uniform."""
    from fastctqw_b200 import graphs
    specs = graphs.uneven_batch(count, seed=seed, nmin=nmin, nmax=nmax)
    As, Xs, P0 = [], [], []
    for sp in specs:
        A = sp.adjacency(np.float32)
        As.append(A)
        Xs.append(np.asarray(1j * A * np.float32(sp.t), dtype=np.complex64))
        P0.append(graphs.uniform_state(sp.n))
    return specs, As, Xs, P0


def bench_batch(args, dev):
    """Grouped batch (one CUDA graph of grouped launches) vs a loop of the per-walk plain form,
    both with the inputs resident in HBM and timed with CUDA events."""
    import torch
    from fastctqw_b200._native import Engine
    from fastctqw_b200.batch import WalkBatch
    specs, As, Xs, P0 = batch_workload(args.batch_count, args.seed, args.batch_nmin, args.batch_nmax)
    ns = [X.shape[0] for X in Xs]
    dX = [torch.from_numpy(X).to(dev) for X in Xs]
    dP0 = [torch.from_numpy(p).to(dev) for p in P0]
    dP = [torch.empty_like(p) for p in dP0]
    stream = torch.cuda.current_stream(dev)
    if args.selector == "learned":
        from fastctqw_b200 import selector as sel
        sel.set_weights()
    reps = max(1, min(args.steps, 3))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(bb):
        for _ in range(max(1, args.warmup)):
            bb.run_device(dX, dP0, dP, stream)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            bb.run_device(dX, dP0, dP, stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / reps

    plain_batch_ms = None
    if args.selector != "plain" or args.form != "plain" or args.approx != "pade":
        bpl = WalkBatch(ns, autotune=not args.no_autotune)
        plain_batch_ms = timed(bpl)
        _, s_plain = bpl.selection()
        bpl.close()
    b = WalkBatch(ns, selector=args.selector, form=args.form, approx=args.approx,
                  autotune=not args.no_autotune)   # tuned in the warm-up
    batch_ms = timed(b)
    info = b.info()
    sched = b.schedule()
    sampled = b.sample_check()
    m, s = b.selection()
    outcome = b.details()["outcome"]
    # accuracy on the largest walks: FP64 eigendecomposition of A on the device
    worst = 0.0
    for k in sorted(range(len(ns)), key=lambda k: -ns[k])[:4]:
        A = torch.from_numpy(As[k]).to(dev, torch.float64)
        lam, V = torch.linalg.eigh(A)
        t32 = float(np.float32(specs[k].t))
        p0 = dP0[k].to(torch.complex128)
        ref = V.to(torch.complex128) @ (torch.exp(1j * lam * t32) * (V.T.to(torch.complex128) @ p0))
        psi = dP[k].to(torch.complex128)
        ov = torch.vdot(ref, psi).abs() ** 2 / (torch.vdot(ref, ref).real * torch.vdot(psi, psi).real)
        worst = max(worst, float(1.0 - ov))
    # | ||psi|| - ||psi0|| | over all walks (U is unitary in exact arithmetic)
    norm_dev = max(abs(float(torch.linalg.vector_norm(p.to(torch.complex128)) - torch.linalg.vector_norm(q.to(torch.complex128))))
                   for p, q in zip(dP, dP0))
    b.close()
    del dP
    # per-walk loop of the plain form (compute only: engines are created outside the timing)
    loop_ms = 0.0
    if not args.no_batch_loop:
        outs = [torch.empty_like(p) for p in dP0]
        for k in range(len(ns)):
            e = Engine(ns[k], np.complex64)
            e.walk_device(dX[k], dP0[k], outs[k], None, stream)   # warm-up of this size
            torch.cuda.synchronize()
            ev0.record(stream)
            e.walk_device(dX[k], dP0[k], outs[k], None, stream)
            ev1.record(stream)
            torch.cuda.synchronize()
            loop_ms += ev0.elapsed_time(ev1)
            e.close()
    walks = len(ns)
    return {
        "workload": f"{walks} walks, N ~ U{{{args.batch_nmin}..{args.batch_nmax}}}, alternating d-regular "
                    f"(d 3..16) / G(N, p 0.05..0.5) adjacency, t log-uniform [0.5, 50], complex64, psi0 uniform",
        "walks_per_s": round(walks / (batch_ms * 1e-3), 1), "ms": round(batch_ms, 2),
        "loop_walks_per_s": round(walks / (loop_ms * 1e-3), 1) if loop_ms else None,
        "loop_ms": round(loop_ms, 1) if loop_ms else None,
        "speedup_vs_loop": round(loop_ms / batch_ms, 2) if loop_ms else None,
        "launches_per_batch": info["launches"], "algorithmic_tflops": round(info["flops"] / (batch_ms * 1e-3) / 1e12, 1),
        "selector": args.selector,
        "form": args.form,
        "approx": args.approx,
        "plain_form_ms": round(plain_batch_ms, 2) if plain_batch_ms else None,
        "plain_form_walks_per_s": round(walks / (plain_batch_ms * 1e-3), 1) if plain_batch_ms else None,
        "squarings_chosen": int(s.sum()), "squarings_plain": int(s_plain.sum()) if plain_batch_ms else None,
        "outcomes": {int(k): int(v) for k, v in zip(*np.unique(outcome, return_counts=True))},
        "m_hist": {int(k): int(v) for k, v in zip(*np.unique(m, return_counts=True))},
        "s_max": int(s.max()), "s_mean": round(float(s.mean()), 2),
        "worst_infidelity_4_largest": worst,
        "norm_deviation_max": norm_dev,
        "sampled_plain_check": sampled,
        "schedule": {"tile_group": sched["tile_group"], "tile_order": sched["tile_order"],
                     "tuned_ms": [[g, o, round(ms, 2)] for g, o, ms in sched["tuned"]]},
    }


def bench_batch_sharded(args, dev, rank, world):
    """The uneven batch sharded over the ranks (longest-processing-time by the cost model, one
    WalkBatch per rank, states gathered on rank 0; fastctqw_b200.shard).  Host buffers in and
    out; wall time between barriers, max over ranks."""
    import torch
    import torch.distributed as dist
    from fastctqw_b200 import shard
    from fastctqw_b200.batch import WalkBatch
    specs, As, Xs, P0 = batch_workload(args.batch_count, args.seed, args.batch_nmin, args.batch_nmax)
    cache = {}

    def runner(xs, ps):
        key = tuple(X.shape[0] for X in xs)
        if key not in cache:
            cache[key] = WalkBatch(list(key), np.complex64, selector=args.selector, form=args.form,
                                   approx=args.approx)
        return cache[key].run(xs, ps)

    if args.selector == "learned":
        from fastctqw_b200 import selector as sel
        sel.set_weights()
    for _ in range(max(1, args.warmup)):
        shard.run_sharded(Xs, P0, runner=runner)
    times = []
    for _ in range(max(1, min(args.steps, 3))):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        shard.run_sharded(Xs, P0, runner=runner)
        torch.cuda.synchronize()
        dist.barrier()
        times.append(time.perf_counter() - t0)
    t = torch.tensor([min(times)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    for b in cache.values():
        b.close()
    ms = float(t.item()) * 1e3
    return {"workload": f"{args.batch_count} uneven walks sharded over {world} ranks (LPT by F(N, m, s))",
            "ms": round(ms, 2), "walks_per_s": round(args.batch_count / (ms * 1e-3), 1),
            "scaling": "strong", "timing": "wall, host buffers in and out, max over ranks"}


def bench_device_setup(args, dev, A: np.ndarray):
    """Walk set-up and read-out on the device against the reference's host steps, at the
    bench's N: X = -1j*H*t from the graph (Operator._buildHamiltonian/_buildUnitory,
    FastCTQW/Operator.py:49-56) and the Hermitian check (:92-103) in numpy on the host, vs
    fx_build_generator from the edge list and fx_check_hermitian on the device; and a 20-point
    time curve at N = 2048 (stepped propagator vs one walk per time)."""
    import time
    import torch
    from fastctqw_b200 import device as fd
    from fastctqw_b200 import graphs
    n, t = A.shape[0], args.t
    t0 = time.perf_counter()
    H = -1.0 * np.asarray(np.diag(A.sum(axis=1)) - A, dtype=np.complex64)
    X_host = np.asarray(-1j * H * t, dtype=np.complex64)
    t1 = time.perf_counter()
    herm_host = bool(np.allclose(H, H.conj().T))
    t2 = time.perf_counter()
    del H
    u, v = np.nonzero(np.triu(A, 1))
    edges = torch.from_numpy(np.stack([u, v], 1).astype(np.int64)).to(dev)
    out = torch.empty((n, n), dtype=torch.complex64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for _ in range(2):
        fd.build_generator(n, edges, t, 1.0, True, np.complex64, out=out)
    torch.cuda.synchronize()
    ev[0].record()
    fd.build_generator(n, edges, t, 1.0, True, np.complex64, out=out)
    ev[1].record()
    herm_dev = fd.is_hermitian(out, skew=True)   # X = -iHt skew-Hermitian <=> H Hermitian
    ev[2].record()
    torch.cuda.synchronize()
    same = bool(np.array_equal(out.cpu().numpy(), X_host))
    del out, edges, X_host
    torch.cuda.empty_cache()
    # time curve: 20 uniform times on G(2048, 0.05), marked nodes 0..7
    from fastctqw_b200.Ctqw import Ctqw
    from fastctqw_b200.State import State
    m = 2048
    Ag = graphs.erdos_renyi(m, 0.05, seed=args.seed, dtype=np.float32)
    adj = [np.nonzero(Ag[i])[0] for i in range(m)]
    w = Ctqw.from_adjacency_list(adj, State.getSingleNodeState(m, 0))
    grid = 0.25 * np.arange(1, 21)
    res = {}
    for method in ("steps", "batch"):
        w.runWalks(grid, list(range(8)), method=method)
        torch.cuda.synchronize()
        s0 = time.perf_counter()
        curve = w.runWalks(grid, list(range(8)), method=method)
        torch.cuda.synchronize()
        res[method] = (round((time.perf_counter() - s0) * 1e3, 2), curve)
    w.free()
    return {
        "n": n, "workload": f"G(n={n}, p=0.5) Laplacian, t={t}, complex64",
        "host_build_X_ms": round((t1 - t0) * 1e3, 1), "host_hermitian_check_ms": round((t2 - t1) * 1e3, 1),
        "device_build_X_ms": round(ev[0].elapsed_time(ev[1]), 3),
        "device_hermitian_check_ms": round(ev[1].elapsed_time(ev[2]), 3),
        "device_X_equals_host_X": same, "hermitian_host_H": herm_host, "skew_hermitian_device_X": herm_dev,
        "time_curve": {"workload": "G(2048, 0.05) adjacency, 20 times 0.25..5.0, 8 marked nodes, complex64",
                       "steps_ms": res["steps"][0], "batch_ms": res["batch"][0],
                       "max_abs_diff": float(np.abs(res["steps"][1] - res["batch"][1]).max())},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=10000)
    ap.add_argument("--t", type=float, default=4.5)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--form", default="mixed", choices=["plain", "mixed", "simt"],
                    help="precision form of the timed walk; the plain form is timed beside it")
    ap.add_argument("--selector", default="estimated", choices=["plain", "certified", "estimated", "learned"],
                    help="(m, s) selection of the timed walk; the plain selection is timed beside it")
    ap.add_argument("--approx", default="chebyshev", choices=["pade", "chebyshev"],
                    help="approximant of the timed walk before its squarings (Pade + solve, or the "
                         "Chebyshev-Bessel polynomial); the plain form beside it is Pade")
    ap.add_argument("--ref-sample-n", type=int, default=1024,
                    help="size of the small sample behind the flop-model cross-check of the reference arm")
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="reference arm: full-size runs are added while their total stays within this")
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 infidelity check")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven-batch leg")
    ap.add_argument("--no-batch-loop", action="store_true", help="skip the per-walk loop of the batch leg")
    ap.add_argument("--batch-only", action="store_true", help="run only the uneven-batch leg")
    ap.add_argument("--no-setup", action="store_true", help="skip the device set-up / time-curve leg")
    ap.add_argument("--no-stress", action="store_true", help="skip the large-norm stress leg (N=16384, t=100)")
    ap.add_argument("--stress-n", type=int, default=16384)
    ap.add_argument("--stress-t", type=float, default=100.0)
    ap.add_argument("--no-autotune", action="store_true", help="batch leg: default schedule, no autotuning")
    ap.add_argument("--batch-shard", action=argparse.BooleanOptionalAction, default=True,
                    help="with N > 1 ranks: also run the uneven batch sharded over the ranks (default on)")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-nmin", type=int, default=64)
    ap.add_argument("--batch-nmax", type=int, default=2048)
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    from fastctqw_b200 import fastexpm
    from fastctqw_b200._native import Engine

    if args.batch_only:
        if rank == 0:
            print(json.dumps({"batch": bench_batch(args, torch.device("cuda", local))}), flush=True)
        return

    n = args.n
    A, H, X = workload(n, args.seed, args.t)
    psi0 = np.zeros(n, dtype=np.complex64)
    psi0[0] = 1.0
    dev = torch.device("cuda", local)
    dX = torch.from_numpy(X).to(dev)
    dpsi0 = torch.from_numpy(psi0).to(dev)
    dpsi = torch.empty_like(dpsi0)
    dU = torch.empty_like(dX)
    if args.selector == "learned":
        from fastctqw_b200 import selector as sel
        sel.set_weights()
    eng = Engine(n, np.complex64)
    eng.configure(form=args.form, selector=args.selector, approx=args.approx)
    stream = torch.cuda.current_stream(dev)

    def step():
        eng.walk_device(dX, dpsi0, dpsi, dU, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # the int8 tensor rate, once here and once after the timed steps (the roofline takes the
    # higher: under the power cap the clock of a short measurement varies from run to run)
    from fastctqw_b200 import _native
    i8_pre = _native.tensor_peak("int8")

    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total_ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    st = eng.stats()
    psi_chosen = dpsi.clone()
    unitarity = None
    if not args.no_check and rank == 0:
        # ||U^H U - I||_F / sqrt(N) of the timed walk's U (complex64 as stored), in complex128
        U128 = dU.to(torch.complex128)
        G = U128.conj().T @ U128
        G.diagonal().sub_(1.0)
        unitarity = float(torch.linalg.matrix_norm(G).item() / np.sqrt(n))
        del U128, G
        torch.cuda.empty_cache()
    if world > 1:
        tt = torch.tensor([total_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms_per_step = total_ms / args.steps
    value = total_ms / (args.steps * world)

    # ---- roofline of the dominant kernel (int8 tensor-core product), timed live in one
    # extra profiled walk with CUDA events around every product launch.
    eng.configure(profile=True)
    step()
    torch.cuda.synchronize()
    pst = eng.stats()
    stages = {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in eng.product_profile().items()}
    timeline = {k: round(v, 3) for k, v in eng.timeline().items()}
    eng.configure(profile=False)
    pk, pk_kind = peaks()
    from fastctqw_b200 import _native
    i8 = _native.tensor_peak("int8")
    bf = _native.tensor_peak("bf16")
    int8_peak = max(i8["tops"], i8_pre["tops"])
    achieved = pst["prod_ops"] / (pst["prod_ms"] * 1e-3) / 1e12 if pst["prod_ms"] > 0 else None
    traffic = product_traffic_per_launch(args.form + ("/chebyshev" if args.approx == "chebyshev" else ""))
    roofline = {
        "bound": "tensor",
        "kernel": ("k_gemm_i8<4,double> (int8 Ozaki-slice products, exact accumulation; 4 slices)"
                   if args.form == "mixed" and args.approx == "chebyshev" else
                   "k_gemm_i8<4,double> and <3,double> (int8 Ozaki-slice products, exact accumulation; "
                   "4 slices, the early Newton-Schulz steps 3)" if args.form == "mixed" else
                   "k_gemm_i8<5,double> (int8 Ozaki-slice product, exact accumulation)"),
        "achieved": round(achieved, 1) if achieved else None, "peak": round(int8_peak, 1), "unit": "TOP/s (int8)",
        "frac": round(achieved / int8_peak, 3) if achieved else None,
        "peak_source": "measured on this GPU by fx_tensor_peak (tcgen05.mma kind::i8 M128 N256, operands in "
                       "shared memory, one CTA per SM, median of 5 launches; the higher of a measurement "
                       "before and one after the timed steps)",
        "peak_measurements": [round(i8_pre["tops"], 1), round(i8["tops"], 1)],
        # under the 1000 W cap the random-operand measurement can run at a lower clock than the
        # products (whose slices toggle fewer bits), so the line also gives the nominal dense int8
        # rate (4.5 POP/s at 1965 MHz) scaled to the median SM clock of the timed steps
        "nominal_at_clock": round(4500.0 * clk["sm_mhz"] / 1965.0, 1) if clk.get("sm_mhz") else None,
        "frac_of_nominal_at_clock": (round(achieved / (4500.0 * clk["sm_mhz"] / 1965.0), 3)
                                     if achieved and clk.get("sm_mhz") else None),
        "traffic": traffic["bytes"] if traffic else None,
        "traffic_source": traffic["source"] if traffic else None,
        "launches": pst["prod_launches"], "kernel_ms_per_walk": round(pst["prod_ms"], 3),
        "kernel_share_of_walk": round(pst["prod_ms"] / ms_per_step, 3),
        "useful_real_tflops": round(pst["prod_flops"] / (pst["prod_ms"] * 1e-3) / 1e12, 2) if pst["prod_ms"] else None,
        "frac_of_2x_bf16": round(achieved / (2.0 * pk["bf16_tflops"]), 3) if achieved else None,
        "bf16_peak_measured_here": round(bf["tops"], 1),
        "bf16_peak_measured_peaks_json": pk.get("bf16_tflops"), "peaks_json": pk_kind,
        "stages": stages,
        "walk_timeline_ms": timeline,
    }

    # ---- the plain form (5-slice products, exact complex squarings) with the plain (Al-Mohy &
    # Higham) selection on the same walk, timed the same way
    plain = None
    psi_plain = None
    if args.selector != "plain" or args.form != "plain" or args.approx != "pade":
        eng.configure(form="plain", selector="plain", approx="pade")
        dU_plain = torch.empty_like(dX)      # dU keeps the timed walk's U for the accuracy check

        def step_plain():
            eng.walk_device(dX, dpsi0, dpsi, dU_plain, stream)
        step_plain()
        torch.cuda.synchronize()
        reps = max(1, min(args.steps, 3))
        ev0.record(stream)
        for _ in range(reps):
            step_plain()
        ev1.record(stream)
        torch.cuda.synchronize()
        pst2 = eng.stats()
        plain = {"ms": round(ev0.elapsed_time(ev1) / reps, 3), "m": pst2["m"], "s": pst2["s"],
                 "steps": reps, "form": "plain", "selector": "plain"}
        psi_plain = dpsi.clone()
        del dU_plain
        torch.cuda.empty_cache()
        eng.configure(form=args.form, selector=args.selector, approx=args.approx)

    # ---- accuracy of both against the FP64 eigendecomposition propagator
    accuracy = None
    if not args.no_check and rank == 0:
        accuracy = accuracy_vs_eigh(H, args.t, dU, psi_chosen, psi_plain, dev, args.seed)
        accuracy["unitarity_residual"] = unitarity

    # ---- end to end through the drop-in API (host ndarray in, host ndarray out)
    e2e = None
    if rank == 0 and not args.no_e2e:
        X_pinned = torch.from_numpy(X).pin_memory().numpy()
        em = fastexpm.ExpMatComplex64(n)
        em.configure(form=args.form, selector=args.selector, approx=args.approx)
        em.run(X_pinned)
        e_steps = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        for _ in range(e_steps):
            Uh = em.run(X_pinned)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / e_steps
        del Uh
        # the same call with an ordinary (pageable) numpy input, as most callers pass it
        em.run(X)
        t0 = time.perf_counter()
        for _ in range(e_steps):
            Uh = em.run(X)
        e2e_pageable_ms = (time.perf_counter() - t0) * 1e3 / e_steps
        em.free()
        e2e = {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(X.nbytes),
               "d2h_bytes_per_step": int(Uh.nbytes), "api": "fastexpm.ExpMatComplex64.run",
               "input": "page-locked numpy array; output a new (pageable) numpy array per call",
               "steps": e_steps, "pageable_input_ms": round(e2e_pageable_ms, 3)}
        del Uh, X_pinned

    # ---- CPU baseline (reference CPU path on this host, bounded sample, rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        times, _ = reference_walks(n, args.seed, args.t, 1, args.ref_budget_s)
        cpu = {"value": round(1e3 * times[0], 1), "unit": "ms", "cores": threads_used(), "kind": "reference",
               "sample": f"one full N={n} walk of the reference CPU path: scipy.linalg.expm(X) + U psi0 "
                         f"(FastCTQW/Operator.py:74-76, Ctqw.py:94) on this host"}

    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        eng.close()
        del dX, dU, dpsi0, dpsi
        torch.cuda.empty_cache()
        batch = bench_batch(args, dev)
    if world > 1 and args.batch_shard:
        if not eng._freed:
            eng.close()
        torch.cuda.empty_cache()
        batch = bench_batch_sharded(args, dev, rank, world)
    stress = None
    if rank == 0 and world == 1 and not args.no_stress:
        if not eng._freed:
            eng.close()
        torch.cuda.empty_cache()
        stress = bench_stress(args, dev)
    setup = None
    if rank == 0 and world == 1 and not args.no_setup:
        if not eng._freed:
            eng.close()
        torch.cuda.empty_cache()
        setup = bench_device_setup(args, dev, A)

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 (int8 Ozaki-slice products, FP64 masters)",
            "data": "synthetic (seeded G(n,0.5) Laplacian)",
            "config": {"workload": f"dense ER G(n={n}, p=0.5) Laplacian, t={args.t}, complex64 expm + U psi0, psi0=|0>",
                       "n": n, "t": args.t, "form": args.form, "selector": args.selector,
                       "approx": args.approx, "degree": st["degree"],
                       "selection_outcome": st["sel_outcome"], "m": st["m"], "s": st["s"],
                       "plain_m": st["plain_m"], "plain_s": st["plain_s"],
                       "solver": {0: "pivoted LU", 1: "cholesky(Q^H Q)", 2: "newton-schulz(Q^H Q)",
                                  3: "none (Chebyshev polynomial)"}[st["solver"]],
                       "l2": "working set ~25 GB >> 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "clocks": clk, "e2e": e2e, "gpu_launches": int(st["launches"]) * args.steps,
            "roofline": roofline, "cpu_baseline": cpu, "accuracy": accuracy, "batch": batch,
            "device_setup": setup, "stress": stress,
            "plain_form": plain,
            "chosen_vs_plain_speedup": round(plain["ms"] / ms_per_step, 3) if plain else None,
            "algorithmic_tflops": round(st["flops"] / (ms_per_step * 1e-3) / 1e12, 2),
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
