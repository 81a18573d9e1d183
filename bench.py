#!/usr/bin/env python
"""Benchmark of the spin-lattice step on B200: atom-steps/s.

Workload (the 4.19M-atom spin-lattice-electron case): bcc Fe, 128^3
conventional cells (4,194,304 atoms), a = 2.8665 A, DD05 EAM + Fe exchange and
Landau terms, Langevin lattice and spin thermostats, localcolmot, electron
temperature on a 16^3 mesh (8^3 unit cells per node) with a Gaussian hot spot
(3,000 K peak, sigma 2 nm, 300 K background), energy renormalisation every
step, dt = 0.5 fs.  Synthetic seeded initial state; spins tilted by a
Gaussian polar angle of 0.35 rad so that the spin temperature starts near
300 K.  The state (about 1 GB) is far larger than L2, so
every step streams it from HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp64|split] [--size 128]

With N > 1 (torchrun) every rank advances its own replica (weak scaling; the
path has no data exchange).  Rank 0 prints one JSON line.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s, 4.19M-atom bcc Fe SLD: split-FP32 vs plain FP64 on one B200"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# Algorithmic HBM bytes per atom and step (compulsory SoA traffic: each
# atom's own state read or written once per pass, neighbour data reused on
# chip).  Per form and pass: bin 28; rho 32 / 16 (FP64 / split); forces (r, s,
# rho in, f out) 80 / 40; four spin visits (r, s, rho in, s out) 4 x 80 / 4 x
# 64; two kicks with the rescale 2 x 120 / 2 x 108; drift 72 / 84.  Totals
# 772 / 640 B per atom-step.
ALGO = {
    "fp64": {"links": 28, "calculate_rho": 32, "calculate_force_energy": 80, "core_ds": 320,
             "core_dp": 240, "core_dr": 72, "step": 772},
    "split": {"links": 28, "calculate_rho": 16, "calculate_force_energy": 40, "core_ds": 256,
              "core_dp": 216, "core_dr": 84, "step": 640},
}
# The bytes this design moves on purpose for core_ds (its visit records and
# exchange rows, which the count above treats as on-chip reuse): a visit
# reads its spin (32 B) and writes it (32 B + the 16 B FP32 copy), reads its
# exchange row (14 pairs x 8 B) and visit record (32 B) = 224 B; backward
# visits also write H, HL and sum J (72 B); 4 visits per step, 2 backward,
# plus the visit records (64 B, twice) = 1,168 B per atom-step.
DESIGN_BYTES_CORE_DS = 1168
# DRAM bytes per atom and step of core_ds measured by ncu at 128^3 (the 72
# k_sweep_pipe launches and the 2 k_spin_noise launches of one step,
# dram__bytes_read.sum + dram__bytes_write.sum, ncu's default cache control:
# caches flushed before every launch, so an upper bound on the graph's own
# traffic); profiles/step_launches_bcc128.md.
CORE_DS_TRAFFIC_PER_ATOM = {"split": (9236.3e6 + 555.8e6) / 4194304,
                            "fp64": (11178.4e6 + 556.0e6) / 4194304}
CORE_DS_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum over one step's 72 "
                          "sweep and 2 visit-record launches at 128^3, caches flushed before "
                          "each launch")
ROOFLINE_KERNEL = {"core_ds": "k_sweep_pipe + k_spin_noise (core_ds: 72 sweep launches "
                              "and 2 visit-record passes per step)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="split", choices=["fp64", "split", "fp64-analytic"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads the default run also measures (64^3 "
                         "Langevin in both forms, the batched replicas, the adjoint)")
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="time only the form given by --precision (the default run also "
                         "times the plain FP64 form on the same state for split / FP64)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in launch shapes instead of sld_autotune's")
    ap.add_argument("--small", action="store_true",
                    help="short run for profiler captures: no CPU baseline, no e2e leg, "
                         "no FP64 arm, no error check, no other workloads, one phase-profile "
                         "step")
    ap.add_argument("--workload", default="single", choices=["single", "replicas", "adjoint"],
                    help="single: the 128^3 spin-lattice-electron system; replicas: many "
                         "independent small systems advanced as one batch; adjoint: gradients "
                         "in the potential's parameters (20^3 cells, NVE)")
    ap.add_argument("--adj-steps", type=int, default=200,
                    help="adjoint workload: trajectory length (steps of 1 fs)")
    ap.add_argument("--adj-checkpoint", type=int, default=20)
    ap.add_argument("--replicas", type=int, default=96)
    ap.add_argument("--out", default=None,
                    help="replicas workload: write per-replica magnetisation vs T here (JSON)")
    return ap.parse_args()


def workload(size, seed=2026):
    from spilady_b200.lattice import hot_spot_te, initial_state
    params, r, p, s = initial_state(size, seed=seed, tilt=0.35, temperature=300.0)
    params["step"] = 0.5e-15
    n_te = max(3, size // 8)
    te = hot_spot_te(n_te, params["box"][0], peak=3000.0, background=300.0, sigma=20.0)
    switches = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True,
                    renormalize=True, te_mesh=n_te)
    return params, r, p, s, te, switches


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ reference
def reference_sample(size, steps, warm, threads):
    """The reference's own CPU build (oracle/_ref) on the benchmark's system:
    bcc Fe size^3 cells, the same physics and start state, Te on the link
    cells (the reference keeps Te per link cell; it has no decoupled mesh).
    ``warm`` untimed steps, then ``steps`` steps timed around core() inside
    the reference's process.  Returns (atom-steps/s, natom, seconds)."""
    from oracle import refjob
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(size, seed=2026, tilt=0.35)
    params["step"] = 0.5e-15
    ops = [(refjob.OP_CORE, warm), (refjob.OP_STATS, 0), (refjob.OP_CORE, steps),
           (refjob.OP_STATS, 0)]
    d = refjob.run("langte", params, r, p, s, ops=ops, threads=threads)[-1]
    return r.shape[0] * steps / d.wall, r.shape[0], d.wall


# The reference's CPU step at 128^3 takes about 11 s on 16 host cores, so its
# timed samples are bounded: the baseline inside our arm times 2 steps after 1
# warm-up step (about 40 s with the set-up); the reference arm times up to
# REF_MAX_STEPS steps after one warm-up step (about 4 min).
REF_MAX_STEPS = 20


def cpu_baseline_block(size, steps=2):
    threads = os.cpu_count() or 1
    from oracle import refjob
    if refjob.available("langte"):
        v, n, t = reference_sample(size, steps, 1, threads)
        return {"value": v, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
                "sample": f"reference CPU build, {size}^3 cells ({n} atoms), {steps} steps "
                          f"after 1 warm-up step, same physics with Te on link cells, "
                          f"{t:.1f} s of core()"}
    return {"value": None, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
            "sample": "reference build absent (oracle/ref/build.sh not run)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, x):
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return x


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import refjob
    if not refjob.available("langte"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build missing (sh oracle/ref/build.sh)"}))
        return
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    warm = 1 if args.warmup > 0 else 0
    v, n, t = reference_sample(args.size, steps, warm, threads)
    line = {"metric": METRIC, "value": v, "unit": "atom-steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * t / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"bcc Fe {args.size}^3 cells ({n} atoms) spin-lattice-electron,"
                                   " Langevin spin+lattice, localcolmot, Te on link cells"
                                   " (the reference has no decoupled Te mesh), dt 0.5 fs",
                       "natom": n, "parallelism": f"OpenMP, {threads} host threads",
                       "steps_note": f"{steps} timed steps (at most {REF_MAX_STEPS}) after "
                                     f"{warm} warm-up step; each step is the whole system"},
            "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{n} atoms x {steps} steps, {t:.1f} s of core()"},
            "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def replicas_cpu_baseline(systems, nrep=4, steps=5):
    """The reference's own CPU build (Langevin spin + lattice) run on the
    first ``nrep`` replicas one after another, ``steps`` steps each after one
    warm-up step: atom-steps/s of the replicas run one by one on the host."""
    from oracle import refjob
    threads = os.cpu_count() or 1
    if not refjob.available("lang"):
        return {"value": None, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
                "sample": "reference build absent (oracle/ref/build.sh not run)"}
    work, secs, edges = 0, 0.0, []
    for edge, temp, params, r, p, s in systems[:nrep]:
        ops = [(refjob.OP_CORE, 1), (refjob.OP_STATS, 0), (refjob.OP_CORE, steps),
               (refjob.OP_STATS, 0)]
        d = refjob.run("lang", params, r, p, s, ops=ops, threads=threads)[-1]
        work += r.shape[0] * steps
        secs += d.wall
        edges.append(edge)
    return {"value": work / secs, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
            "sample": f"reference CPU build (Langevin spin + lattice), replicas of edges {edges} "
                      f"one after another, {steps} steps each after 1 warm-up step"}


def adjoint_cpu_baseline(params, r, p, s, K, nparam=36, steps=10):
    """What a gradient by central differences of the reference's own CPU code
    costs: 2 x nparam K-step NVE trajectories of its param build (the
    potential's constants read from a file), estimated from ``steps`` timed
    steps after one warm-up step.  Returns ms per gradient."""
    from oracle import refjob
    threads = os.cpu_count() or 1
    if not refjob.available("param"):
        return {"value": None, "unit": "ms", "cores": threads, "kind": "reference",
                "sample": "reference build absent (oracle/ref/build.sh not run)"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import DEFAULT_THETA
    ops = [(refjob.OP_CORE, 1), (refjob.OP_STATS, 0), (refjob.OP_CORE, steps), (refjob.OP_STATS, 0)]
    d = refjob.run("param", params, r, p, s, ops=ops, threads=threads,
                   inputs={"theta.in": " ".join("%.17g" % x for x in DEFAULT_THETA)})[-1]
    per_step = d.wall / steps
    return {"value": 2 * nparam * K * per_step * 1e3, "unit": "ms", "cores": threads,
            "kind": "reference",
            "sample": f"reference CPU build (param, NVE), {r.shape[0]} atoms, {steps} timed steps "
                      f"({per_step * 1e3:.1f} ms each) x {2 * nparam} trajectories x {K} steps"}


def replicas_workload(n, seed=2027):
    """n independent bcc Fe boxes: cubic edge uniform on 8..32 cells,
    temperature uniform on 100..1200 K, Langevin spin and lattice
    thermostats, dt 1 fs, each with its own Philox stream (replica k)."""
    from spilady_b200.lattice import initial_state
    rng = np.random.default_rng(seed)
    edges = rng.integers(8, 33, size=n)
    temps = rng.uniform(100.0, 1200.0, size=n)
    out = []
    for k in range(n):
        params, r, p, s = initial_state(int(edges[k]), seed=seed + 1 + k, tilt=0.05,
                                        temperature=float(temps[k]))
        params["temperature"] = float(temps[k])
        params["step"] = 1e-15
        out.append((int(edges[k]), float(temps[k]), params, r, p, s))
    return out


def run_replicas(args, world, rank, local):
    from spilady_b200 import engine
    import torch
    torch.cuda.set_device(local)
    prec = {"fp64": engine.FP64, "split": engine.SPLIT,
            "fp64-analytic": engine.FP64_ANALYTIC}[args.precision]
    sw = dict(spinlang=True, lattlang=True)
    systems = replicas_workload(args.replicas, seed=2027 + 1000 * rank)
    engines = [engine.Engine(params, r, p, s, device=local, precision=prec, replica=k, **sw)
               for k, (edge, temp, params, r, p, s) in enumerate(systems)]
    natom = sum(e.natom for e in engines)
    batch = engine.Batch(engines)
    batch.run(args.warmup)
    for e in engines:
        e.sync()
    clocks = ClockSampler(local)
    barrier(world)
    clocks.start()
    batch.run(args.steps)
    ms = batch.last_run_ms()
    clk = clocks.stop()
    ms = allmax(world, ms)
    value = natom * args.steps * world / (ms / 1e3)
    # the same replicas one after another, each its own graph replays
    seq_ms = 0.0
    for e in engines:
        e.run(args.steps)
        e.sync()
        seq_ms += e.last_run_ms()
    seq_ms = allmax(world, seq_ms)
    per = []
    for (edge, temp, *_), e in zip(systems, engines):
        a = e.averages()
        per.append({"edge": edge, "natom": e.natom, "T_K": temp, "Tl_K": a["Tl"],
                    "m": float(np.sqrt(a["sx"] ** 2 + a["sy"] ** 2 + a["sz"] ** 2))})
    kernels = sum(e.step_kernel_count() for e in engines)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = replicas_cpu_baseline(systems)
    batch.close()
    for e in engines:
        e.close()
    if args.out and rank == 0:
        with open(args.out, "w") as fh:
            json.dump({"steps": args.warmup + 2 * args.steps, "replicas": per}, fh, indent=1)
    if rank != 0:
        return
    line = {
        "metric": f"atom-steps/s, {args.replicas} replicas of bcc Fe (edges 8-32 cells), "
                  "batched in one graph per step",
        "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec == engine.SPLIT else "f64", "data": "synthetic",
        "config": {"workload": f"{args.replicas} independent bcc Fe boxes, edge U{{8..32}} cells, "
                               "T U[100,1200] K, Langevin spin+lattice, dt 1 fs, own Philox "
                               "stream each", "natom": natom, "precision": args.precision,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "one_by_one": {"value": natom * args.steps * world / (seq_ms / 1e3),
                       "ms_per_step": seq_ms / args.steps,
                       "how": "each replica's own graph replays, one replica after another"},
        "roofline": None, "cpu_baseline": cpu, "e2e": None,
        "gpu_launches": kernels * args.steps, "clocks": clk,
    }
    print(json.dumps(line))


def run_adjoint(args, world, rank, local):
    """Gradients of E and of L = sum |f|^2 + |H|^2 in the 36 potential
    parameters: bcc Fe 20^3 cells (16,000 atoms), positions displaced by a
    Gaussian of 0.05 A, spins tilted by 0.2 rad, NVE, dt 1 fs; one
    configuration, then through args.adj_steps steps with a checkpoint every
    args.adj_checkpoint steps; each gradient against FP64 central finite
    differences (h = 1e-6 of each parameter)."""
    from spilady_b200 import engine
    from spilady_b200.lattice import initial_state
    import torch
    torch.cuda.set_device(local)
    if rank != 0:
        return
    prec = {"fp64": engine.FP64, "split": engine.SPLIT,
            "fp64-analytic": engine.FP64_ANALYTIC}[args.precision]
    params, r, p, s = initial_state(20, seed=2029, tilt=0.2, temperature=300.0, pos_sigma=0.05)
    params["step"] = 1e-15
    e = engine.Engine(params, r, p, s, device=local, precision=prec)
    th = engine.adjoint_theta_default()
    h = np.where(th != 0.0, 1e-6 * np.abs(th), 1e-6)
    K, C = args.adj_steps, args.adj_checkpoint

    def timed(fn, reps):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            out = fn()
        return out, (time.perf_counter() - t0) / reps * 1e3

    (cfg, ms_cfg) = timed(lambda: e.adjoint_config(th), 3)
    out, dE, dL = cfg
    ((Lk, dLk), ms_traj) = timed(lambda: e.adjoint_trajectory(th, K, C), 3)
    (_, ms_fwd) = timed(lambda: e.adjoint_trajectory(th, K, C, grad=False), 3)

    def fd(fn, scale=1.0):
        g = np.zeros(len(th))
        for k in range(len(th)):
            tp, tm = th.copy(), th.copy()
            tp[k] += scale * h[k]
            tm[k] -= scale * h[k]
            g[k] = (fn(tp) - fn(tm)) / (2 * scale * h[k])
        return g

    def err(g, f):
        scale = np.max(np.abs(f))
        return float(np.max(np.abs(g - f)) / scale)

    # finite differences of the FP64 model (the split forward's FP32 rounding
    # would swamp differences of 1e-6 in the parameters)
    e64 = engine.Engine(params, r, p, s, device=local, precision=engine.FP64_ANALYTIC)
    fdE = fd(lambda t: e64.adjoint_config(t)[0][0])
    fdL = fd(lambda t: e64.adjoint_config(t)[0][1])
    fdT = fd(lambda t: e64.adjoint_trajectory(t, K, C, grad=False))
    # A sharper check of the trajectory gradient.  Through 200 steps the
    # rounding of every step is amplified with the trajectory's separation,
    # which makes L(theta) noisy on the scale of h = 1e-6; central differences
    # with 100x larger steps (1e-4 and 5e-5 of each parameter) see 100x less of
    # that noise, and Richardson's extrapolation of the two removes their
    # O(h^2) truncation error.
    fdA = fd(lambda t: e64.adjoint_trajectory(t, K, C, grad=False), 100.0)
    fdB = fd(lambda t: e64.adjoint_trajectory(t, K, C, grad=False), 50.0)
    fdTR = (4.0 * fdB - fdA) / 3.0
    _, dLk64 = e64.adjoint_trajectory(th, K, C)
    cpu = None if args.no_cpu_baseline else adjoint_cpu_baseline(params, r, p, s, K)
    line = {
        "metric": f"ms per gradient of L in 36 potential parameters through {K} NVE steps, "
                  f"{e.natom}-atom bcc Fe",
        "value": ms_traj, "unit": "ms", "n_gpus": 1, "steps": K, "warmup": 1,
        "ms_per_step": ms_traj / max(K, 1), "higher_is_better": False, "scaling": None,
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"bcc Fe 20^3 cells ({e.natom} atoms), positions +N(0, 0.05 A), "
                               f"spin tilt 0.2 rad, NVE dt 1 fs, {K} steps, checkpoint every {C}",
                   "forward_precision": args.precision},
        "forward_ms": ms_fwd, "config_gradient_ms": ms_cfg,
        "E": out[0], "L": out[1], "L_final": Lk,
        "vs_finite_differences": {"dE_config": err(dE, fdE), "dL_config": err(dL, fdL),
                                  f"dL_{K}_steps": err(dLk, fdT),
                                  f"dL_{K}_steps_fp64_forward": err(dLk64, fdT),
                                  f"dL_{K}_steps_fp64_forward_vs_richardson": err(dLk64, fdTR),
                                  f"dL_{K}_steps_vs_richardson": err(dLk, fdTR),
                                  "fd_h_vs_richardson": err(fdT, fdTR),
                                  "how": "max |adjoint - FD| / max |FD| over the 36 parameters; "
                                         "FD: FP64 central differences, h = 1e-6 relative; "
                                         "richardson: from h = 1e-4 and 5e-5 relative"},
        "roofline": None, "cpu_baseline": cpu, "e2e": None,
    }
    print(json.dumps(line))


def other_configs(local):
    """The other workloads, measured briefly in the default run (each device-
    timed with CUDA events on its engine's stream):
      - 64^3 cells (524,288 atoms), Langevin spin and lattice thermostats at
        300 K, dt 1 fs, 1,000 steps in each form, with the split form's error
        against the FP64 form on the start state and their averages at the end;
      - 96 replicas (edges 8-32 cells, 100-1,200 K, Langevin), 20 steps batched
        in one graph per step and 20 steps one replica after another;
      - the adjoint: the gradient of L in the 36 potential parameters through
        200 NVE steps of a 20^3-cell box (split forward), and its error against
        FP64 central differences through 10 steps."""
    from spilady_b200 import engine
    from spilady_b200.lattice import initial_state
    out = {}
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    # 64^3 Langevin
    params, r, p, s = initial_state(64, seed=2028, tilt=0.05, temperature=300.0)
    params["step"] = 1e-15
    sw = dict(spinlang=True, lattlang=True)
    n_steps = 1000
    res, start = {}, {}
    for name, form in (("split", engine.SPLIT), ("fp64", engine.FP64)):
        e = engine.Engine(params, r, p, s, device=local, precision=form, **sw)
        start[name] = {n: e.get(n) for n in ("f", "rho", "pe", "me")}
        e.run(n_steps)
        e.sync()
        ms = e.last_run_ms()
        a = e.averages()
        res[name] = {"value": e.natom * n_steps / (ms / 1e3), "ms_per_step": ms / n_steps,
                     "Tl_K": a["Tl"], "m": float(np.sqrt(a["sx"] ** 2 + a["sy"] ** 2 + a["sz"] ** 2)),
                     "pe": a["pe"], "me": a["me"]}
        e.close()
    out["bcc64_langevin"] = {
        "workload": "bcc Fe 64^3 cells (524288 atoms), Langevin spin (gamma 0.01) and lattice "
                    "(1/ps) thermostats at 300 K, dt 1 fs, 1000 steps, first step included",
        "unit": "atom-steps/s", "split": res["split"], "fp64": res["fp64"],
        "split_over_fp64": res["split"]["value"] / res["fp64"]["value"],
        "split_error_start": dict(
            {n: rel(start["split"][n], start["fp64"][n]) for n in start["fp64"]},
            f_abs_eV_per_A=float(np.max(np.abs(start["split"]["f"] - start["fp64"]["f"]))),
            how="max |split - fp64| / max |fp64| on the perfect-lattice start state, whose "
                "net forces nearly vanish by symmetry (so f_abs is given too)"),
        "split_vs_fp64_averages_at_end": {
            q: abs(res["split"][q] - res["fp64"][q]) / abs(res["fp64"][q])
            for q in ("Tl_K", "m", "pe", "me")}}
    # replicas
    systems = replicas_workload(96)
    engines = [engine.Engine(pr, rr, pp, ss, device=local, precision=engine.SPLIT, replica=k, **sw)
               for k, (edge, temp, pr, rr, pp, ss) in enumerate(systems)]
    natom = sum(e.natom for e in engines)
    batch = engine.Batch(engines)
    batch.run(3)
    batch.run(20)
    ms = batch.last_run_ms()
    seq = 0.0
    for e in engines:
        e.run(20)
        e.sync()
        seq += e.last_run_ms()
    batch.close()
    for e in engines:
        e.close()
    out["replicas"] = {"workload": f"96 bcc Fe boxes ({natom} atoms), edges 8-32 cells, 100-1200 K, "
                                   "Langevin spin + lattice, dt 1 fs, split form, 20 steps",
                       "unit": "atom-steps/s", "batched": natom * 20 / (ms / 1e3),
                       "one_by_one": natom * 20 / (seq / 1e3)}
    # adjoint
    params, r, p, s = initial_state(20, seed=2029, tilt=0.2, temperature=300.0, pos_sigma=0.05)
    params["step"] = 1e-15
    es = engine.Engine(params, r, p, s, device=local, precision=engine.SPLIT)
    e64 = engine.Engine(params, r, p, s, device=local, precision=engine.FP64_ANALYTIC)
    th = engine.adjoint_theta_default()
    es.adjoint_trajectory(th, 200, 20)
    grad_runs = []
    for _ in range(3):   # the median of three: host-timed, so it varies from run to run
        t0 = time.perf_counter()
        es.adjoint_trajectory(th, 200, 20)
        grad_runs.append((time.perf_counter() - t0) * 1e3)
    grad_ms = float(np.median(grad_runs))
    K = 10
    _, g = e64.adjoint_trajectory(th, K, 5)
    h = np.where(th != 0.0, 1e-6 * np.abs(th), 1e-6)
    fd = np.zeros(len(th))
    for k in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[k] += h[k]
        tm[k] -= h[k]
        fd[k] = (e64.adjoint_trajectory(tp, K, 5, grad=False) -
                 e64.adjoint_trajectory(tm, K, 5, grad=False)) / (2 * h[k])
    es.close()
    e64.close()
    out["adjoint"] = {"workload": "gradient of L = sum |f|^2 + |H|^2 in 36 potential parameters, "
                                  "bcc Fe 20^3 cells (16000 atoms), NVE dt 1 fs",
                      "ms_per_gradient_200_steps_split_forward": grad_ms,
                      "error_vs_fd_10_steps": float(np.max(np.abs(g - fd)) / np.max(np.abs(fd))),
                      "how": "max |adjoint - FD| / max |FD|; FD: FP64 central differences, "
                             "h = 1e-6 relative, on the FP64 analytic model"}
    return out


def main():
    args = parse()
    if args.small:
        args.no_cpu_baseline = True
        args.no_e2e = True
        args.no_configs = True
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "replicas":
        run_replicas(args, world, rank, local)
        return
    if args.workload == "adjoint":
        run_adjoint(args, world, rank, local)
        return
    from spilady_b200 import engine
    import torch
    torch.cuda.set_device(local)
    params, r, p, s, te, sw = workload(args.size)
    forms = {"fp64": engine.FP64, "split": engine.SPLIT, "fp64-analytic": engine.FP64_ANALYTIC}
    prec = forms[args.precision]
    # The split form's error against the FP64 run of the same kernels and
    # against the reference's arithmetic (the FP64 form), on the start state:
    # forces, exchange fields and per-atom energies (held to 1e-5 relative).
    split_err = None
    if prec == engine.SPLIT and not args.small:
        e = engine.Engine(params, r, p, s, te=te, device=local, precision=prec, **sw)
        ref = engine.Engine(params, r, p, s, te=te, device=local, precision=engine.FP64, **sw)
        rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
        split_err = {q: rel(e.get(n), ref.get(n)) for q, n in
                     (("force", "f"), ("field", "H"), ("rho", "rho"), ("pe", "pe"),
                      ("me", "me"))}
        split_err["force_abs_eV_per_A"] = float(np.max(np.abs(e.get("f") - ref.get("f"))))
        split_err["how"] = ("max |split - fp64| / max |fp64| over all atoms, start state; the "
                            "FP64 form is the reference's arithmetic (its tables)")
        ref.close()
        e.close()

    def timed_form(form, with_e2e):
        """One form: autotune, warm up, time args.steps graph steps (CUDA
        events on the engine stream), profile the phases; optionally the e2e
        leg through the public API.  Returns a dict."""
        e = engine.Engine(params, r, p, s, te=te, device=local, precision=form, **sw)
        shapes = None if args.no_autotune else e.autotune(steps=12)
        e.run(args.warmup)
        e.sync()
        clocks = ClockSampler(local)
        barrier(world)
        torch.cuda.synchronize()
        clocks.start()
        e.run(args.steps)
        ms = e.last_run_ms()
        torch.cuda.synchronize()
        barrier(world)
        clk = clocks.stop()
        e.sync()
        ms = allmax(world, ms)
        out = {"ms": ms, "value": e.natom * args.steps * world / (ms / 1e3), "clocks": clk,
               "shapes": shapes, "kernels_per_step": e.step_kernel_count(), "natom": e.natom}
        prof = {}
        nprof = 1 if args.small else 5
        for _ in range(nprof):
            for k, v in e.profile_step().items():
                prof[k] = prof.get(k, 0.0) + v / nprof
        out["prof"], out["nprof"] = prof, nprof
        if with_e2e:
            out["e2e"] = e2e_leg(e)
        e.close()
        return out

    def e2e_leg(e):
        # End to end through the public API with host buffers: upload the
        # state from pinned host memory (sld_set_state), then every step run
        # it and read the check() averages back, as the reference's main loop
        # prints them every step at interval_of_print_out 1, and at the end of
        # the sample read the whole configuration (r, p, s) back into the
        # pinned buffers, as a configuration file written every k steps
        # needs.  The state stays on the device between steps, as it does
        # behind the reference's core() with a device backend.
        host = {}
        for name, a in (("r", r), ("p", p), ("s", s)):
            host[name] = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            host[name].numpy()[:] = a
        k = max(5, min(args.steps, 100))
        secs = []
        for _ in range(3):   # three samples, the median: the host's own timing varies
            t0 = time.perf_counter()
            e.set_state(host["r"].numpy(), host["p"].numpy(), host["s"].numpy())
            for _ in range(k):
                e.run(1)
                e.averages()
            for name in ("r", "p", "s"):
                e.get(name, out=host[name].numpy().reshape(-1))
            secs.append(time.perf_counter() - t0)
        nat = e.natom
        return {"value": nat * k / float(np.median(secs)), "unit": "atom-steps/s",
                "h2d_bytes_per_step": int(nat * 72 / k),
                "d2h_bytes_per_step": int(80 + nat * 72 / k), "steps": k,
                "note": f"per sample of {k} steps: r, p, s uploaded from pinned host memory "
                        "once (sld_set_state), sld_run(1) and the averages read back every "
                        "step, and r, p, s read back into the pinned buffers at the end; "
                        "the median of three samples"}

    main_arm = timed_form(prec, not args.no_e2e)
    fp64_arm = None
    if prec == engine.SPLIT and not (args.no_fp64_arm or args.small):
        fp64_arm = timed_form(engine.FP64, False)
    natom = main_arm["natom"]
    ms, value, prof, nprof = main_arm["ms"], main_arm["value"], main_arm["prof"], main_arm["nprof"]
    key = "split" if prec == engine.SPLIT else "fp64"
    dom = max((k for k in prof if k in ALGO[key]), key=prof.get)
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = ALGO[key][dom] * natom / (prof[dom] / 1e3) / 1e9 if prof[dom] > 0 else 0.0
    traffic = None
    if dom == "core_ds" and key in CORE_DS_TRAFFIC_PER_ATOM:
        traffic = CORE_DS_TRAFFIC_PER_ATOM[key] * natom
    step_achieved = ALGO[key]["step"] * natom / (ms / args.steps / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": ROOFLINE_KERNEL.get(dom, dom), "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "per": "one step of the phase (algorithmic bytes and traffic per step)",
                "algorithmic_bytes": ALGO[key][dom] * natom,
                "algorithmic_bytes_per_atom": ALGO[key][dom],
                "traffic_source": CORE_DS_TRAFFIC_SOURCE if traffic else None,
                "design_bytes": {"per_atom": DESIGN_BYTES_CORE_DS,
                                 "achieved": DESIGN_BYTES_CORE_DS * natom / (prof[dom] / 1e3) / 1e9,
                                 "what": "core_ds with this design's visit records and "
                                         "exchange rows counted"} if dom == "core_ds" else None,
                "whole_step": {"bytes_per_atom": ALGO[key]["step"], "achieved": step_achieved,
                               "frac": step_achieved / hbm},
                "peak_source": "measured (burst copy)" if peaks else "fallback",
                "timing": f"CUDA events around each phase on the engine stream, {nprof} "
                          "sequential steps after the timed region",
                "phase_ms": {k: round(v, 4) for k, v in prof.items()}}
    fp64_block = None
    if fp64_arm is not None:
        fp64_block = {"value": fp64_arm["value"], "ms_per_step": fp64_arm["ms"] / args.steps,
                      "phase_ms": {k: round(v, 4) for k, v in fp64_arm["prof"].items()},
                      "launch_shapes": fp64_arm["shapes"], "clocks": fp64_arm["clocks"],
                      "how": "the plain FP64 form (the reference's arithmetic) on the same "
                             "state, box and steps, timed the same way"}

    if rank != 0:
        return
    configs = None
    if world == 1 and not args.no_configs:
        configs = other_configs(local)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(args.size)
    line = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec == engine.SPLIT else "f64",
        "data": "synthetic",
        "config": {"workload": f"bcc Fe {args.size}^3 cells ({natom} atoms) spin-lattice-electron,"
                               f" Langevin spin+lattice, localcolmot, Te mesh {sw['te_mesh']}^3,"
                               " dt 0.5 fs",
                   "precision": args.precision, "natom": natom,
                   "l2": "state (~3 GB) larger than L2; no flush needed",
                   "launch_shapes": main_arm["shapes"],
                   "split_error": split_err,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "fp64": fp64_block,
        "split_over_fp64": (value / fp64_arm["value"]) if fp64_arm else None,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": main_arm.get("e2e"),
        "gpu_launches": main_arm["kernels_per_step"] * args.steps, "clocks": main_arm["clocks"],
        "other_workloads": configs,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
