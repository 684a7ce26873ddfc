#!/usr/bin/env python
"""Benchmark of the pressure-equation hot path on B200.

Workload (one step = one pressure solve): the 3D Taylor-Green vortex pressure equation on the
periodic box [0,2pi]^3 with a uniform 128^3 hex mesh (2,097,152 cells, 6,291,456 faces), as the
PIMPLE corrector assembles it: fvm::laplacian(rAUf, p) with rAUf = dt = 2e-3, minus the divergence
of a predicted face flux phi = (u_TG + seeded perturbation)_f . S_f, setReference(cell 0), solved
from p = 0 with PCG + GAMG to relTol 1e-8 (tolerance 0, the reference's normalised L1 residual).
Synthetic data: the TG field plus 16 seeded Fourier modes (|k| <= 4, amplitude N(0,1)/|k|^2).

Metric: solves/s (whole job, all GPUs) and p50/p99 latency, mixed precision (FP32 GAMG V-cycle
inside the FP64 PCG recurrence) vs FP64 GAMG-PCG.  `value` is the mixed-precision rate with inputs
resident in HBM; `e2e` is the same through the host-pointer C ABI (vlm_ldu_solve: H2D of
diag/upper/b/x and D2H of x inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 128]

--workload serving: a seeded Poisson trace of steady lid-cavity solves through the serving runtime
(vlm_server_*), mixed-precision vs FP64 pressure, solves/s and p50/p99 latency; --impl reference
replays the trace through the reference's own incompressible solver in host worker processes.

--workload batch [--systems 256]: config 3, a batch of uneven graded, jittered Poisson systems solved
in one batched pressure corrector (nNonOrthCorr 2, FP32 V-cycles in FP64 PCG), systems/s; the
reference arm times the reference's pressure loop on the batch's first --ref-systems systems.

--workload channel [--channel 256x192x128]: the Re_tau 395 LES channel (Smagorinsky + Van Driest,
mean-velocity forcing), PIMPLE steps/s with mixed vs FP64 pressure; --impl reference times the
reference's own LES step on a 96x72x48 sample and scales it by cells.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 2e-3
REL_TOL = 1e-8


# ------------------------------------------------------------------------------ replicas (N > 1)
def max_over_ranks(value, world, device=None):
    """The largest of one float per rank (a multi-GPU time is the slowest rank's); every rank takes
    this collective in the same order.  device: the tensor's device (CUDA for NCCL, None for gloo)."""
    if world <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def deal(items, rank, world):
    """Replica sharding: item i goes to rank i mod world (no item twice, none lost)."""
    return list(items)[rank::world]


def aggregate_rate(units_per_rank, world, seconds):
    """Whole-job throughput of `world` replicas that each processed units_per_rank in (max) seconds."""
    return world * units_per_rank / seconds


# ------------------------------------------------------------------------------ workload
def tg_velocity(C, seed=1234, n_modes=16, amp=0.1):
    x, y, z = C[:, 0], C[:, 1], C[:, 2]
    u = np.stack([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), np.zeros_like(x)], 1)
    rng = np.random.default_rng(seed)
    for _ in range(n_modes):
        k = rng.integers(-4, 5, size=3)
        if not k.any():
            k[0] = 1
        kk = float(np.sqrt((k * k).sum()))
        a = rng.standard_normal(3) / kk ** 2
        ph = rng.uniform(0, 2 * np.pi)
        u += amp * np.outer(np.cos(C @ k + ph), a)
    return u


def assemble(m):
    """LDU pressure system from cfd::Mesh arrays: laplacian(rAUf=DT) (Fvm.h:149-154), source +=
    divPhi*V (FvMatrix.h:93-97 via Fvc.h:294-304), setReference(0) (FvMatrix.h:134-141)."""
    nC, nI = m["n_cells"], len(m["neighbour"])
    own, nei = m["owner"][:nI], m["neighbour"]
    upper = DT * m["magSf"][:nI] * m["ndc"][:nI]
    diag = np.zeros(nC)
    np.subtract.at(diag, np.stack([own, nei], 1).ravel(), np.repeat(upper, 2))
    u = tg_velocity(m["C"])
    w = m["w"][:nI, None]
    uf = w * u[own] + (1.0 - w) * u[nei]
    Sf = m["Sf"][:nI]
    phi = uf[:, 0] * Sf[:, 0] + uf[:, 1] * Sf[:, 1] + uf[:, 2] * Sf[:, 2]
    div = np.zeros(nC)
    np.add.at(div, np.stack([own, nei], 1).ravel(), np.stack([phi, -phi], 1).ravel())
    b = (div / m["V"]) * m["V"]
    b[0] += diag[0] * 0.0
    diag[0] += diag[0]
    return diag, upper, b


def our_mesh(n):
    from voluma_b200 import mesh as vm
    return vm.box_mesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))


def ref_mesh_arrays(n):
    from oracle import ref
    R = ref.RefMesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    m = {k: R.get(k) for k in ("owner", "neighbour", "magSf", "ndc", "C", "w", "Sf", "V")}
    m["n_cells"] = R.n_cells
    return R, m


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi's clock and throttle-reason record during a timed region: one nvidia-smi process
    streaming a line every 20 ms (-lms), started before the region (start() returns once the first
    line has arrived) and ended after it by its own PID."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.samples = []
        self._proc = None
        self._t = None
        self._first = threading.Event()

    def start(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", "20"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._proc = None
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        self._first.wait(timeout=5.0)

    def _run(self):
        for line in self._proc.stdout:
            out = line.strip()
            if out:
                self.samples.append([v.strip() for v in out.split(",")])
                self._first.set()

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except Exception:
                self._proc.kill()
        if self._t:
            self._t.join(timeout=10)
        # the samples of the timed region: drop the one that start() waited for
        samples = self.samples[1:] if len(self.samples) > 1 else self.samples
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if len(s) > 4 + i and
                          s[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel, n):
    """dram bytes per launch of `kernel` at n^3 from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    try:
        for line in open(p):
            f = line.split()
            if len(f) >= 3 and f[0] == kernel and int(f[1]) == n:
                return float(f[2])
    except Exception:
        pass
    return None


# ------------------------------------------------------------------------------ reference arm
def pressure_config(n, world, smoother=""):
    """The config dict of the pressure workload, the same keys in both arms."""
    return {"workload": f"TGV {n}^3 periodic pressure equation (laplacian(rAUf) - div(phiHbyA), setReference), "
                        f"PCG+GAMG relTol 1e-8 from p=0", "cells": n ** 3, "faces": 3 * n ** 3,
            "smoother": smoother or "mcgs-jacobi", "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (matrix hierarchy + vectors > 126 MB)"}


def _ref_worker(n, nsolves, barrier, out):
    """One single-threaded reference process: builds the mesh, the system and the cached GAMG hierarchy
    (untimed), waits for every process, then runs its share of the solves back to back."""
    sys.path.insert(0, ROOT)
    R, m = ref_mesh_arrays(n)
    diag, upper, b = assemble(m)
    R.gamg_levels()  # builds and caches the hierarchy (GAMG.cpp:204) outside the timed solves
    barrier.wait()
    t0 = time.time()
    times, iters = [], []
    for _ in range(nsolves):
        t = time.perf_counter()
        _, perf = R.solve(diag, upper, None, b, np.zeros(m["n_cells"]), "PCG", "GAMG", 0.0, REL_TOL, 1000)
        times.append(time.perf_counter() - t)
        iters.append(perf["iterations"])
    out.put((t0, time.time(), times, iters))


def run_reference(args, rank, world):
    """The reference's own solveLdu (PCG + its GS-smoothed GAMG, compiled from its sources) on the same
    system: exactly `steps` solves dealt over single-threaded processes, one per host core (up to
    `steps`); throughput = steps / wall time from the common start to the last solve's end."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvlmref.so was not built (make -C oracle)"}))
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    P = max(1, min(cores, args.steps))
    share = [args.steps // P + (1 if i < args.steps % P else 0) for i in range(P)]
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(P), ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=(args.n, share[i], barrier, out)) for i in range(P)]
    for q in procs:
        q.start()
    res = [out.get() for _ in procs]
    for q in procs:
        q.join()
    wall = max(r[1] for r in res) - min(r[0] for r in res)
    times = [t for r in res for t in r[2]]
    iters = [i for r in res for i in r[3]]
    value = len(times) / wall
    line = {"metric": METRIC, "impl": "reference", "unit": "solves/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup, "value": value,
            "ms_per_step": 1e3 * wall / len(times), "p50_ms": 1e3 * float(np.percentile(times, 50)),
            "p99_ms": 1e3 * float(np.percentile(times, 99)), "iterations": int(np.median(iters)), "dtype": "f64",
            "data": "synthetic", "scaling": "weak", "vs_baseline": None,
            "config": dict(pressure_config(args.n, 1, args.smoother), processes=P, host_cores=cores,
                           smoother="reference GaussSeidel GAMG (GAMG.cpp:363-385)"),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": P, "kind": "reference",
                             "sample": f"{len(times)} full solves dealt over {P} single-threaded processes on "
                                       f"{cores} host cores (reference solveLdu PCG+GAMG, hierarchy pre-built); "
                                       f"wall {wall:.1f} s from the common start"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ serving workload
SERVE_METRIC = "serving: steady lid-cavity SIMPLE solves/s and p50/p99 latency (residualTol 1e-6)"


def serve_trace(args):
    from voluma_b200 import cases
    return cases.serving_trace(args.requests, args.rate, seed=20261203, n_range=(args.nmin, args.nmax),
                               re_range=(args.remin, args.remax))


def serve_config(args, world):
    return {"workload": f"Poisson arrivals ({args.rate}/s) of steady 2D lid-driven cavity solves, N^2 cells with N "
                        f"uniform in {{{args.nmin}..{args.nmax}}}, Re uniform in [{args.remin}, {args.remax}], lid U=1, "
                        f"SIMPLE (linearUpwind, alphaU 0.7, alphaP 0.3, PBiCGStab/DILU U, PCG/GAMG p) to residualTol "
                        f"1e-6; trace seed 20261203",
            "requests": args.requests, "rate_hz": args.rate, "n_range": [args.nmin, args.nmax],
            "re_range": [args.remin, args.remax], "max_active": args.max_active, "hbm_budget_gb": args.hbm_gb,
            "parallelism": f"replicas{world}", "latency": "arrival to completion, server clock (wall)",
            "l2": "each request's working set is small; requests overlap on the device"}


def _serve_ref_worker(q):
    sys.path.insert(0, ROOT)
    from oracle import ref
    from voluma_b200 import cases
    m, case = cases.lid_cavity(q["n"], q["Re"])
    t = time.perf_counter()
    R = ref.RefMesh((q["n"], q["n"], 1), hi=(1.0, 1.0, 0.1), two_d=True)
    _, _, _, hist = R.flow_run(case, 20000, residual_tol=1e-6)
    return time.perf_counter() - t, len(hist)


def run_serving_reference(args, rank, world):
    """The same trace replayed on the host: the reference's IncompressibleFlow (generateBox + Mesh::build +
    the steady loop) in single-threaded worker processes, one per host core.  Each request is submitted
    at its arrival time on the wall clock and its latency is measured from arrival to completion."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvlmref.so was not built (make -C oracle)"}))
        return
    import multiprocessing as mp
    trace = serve_trace(args)
    cores = os.cpu_count() or 1
    P = max(1, min(cores, len(trace)))
    done = {}
    with mp.get_context("spawn").Pool(P) as pool:
        pool.map(_serve_ref_idle, range(P))  # workers started and the reference library loaded
        t0 = time.time() + 0.05
        pending = []
        for i, q in enumerate(trace):
            wait = t0 + q["arrival"] - time.time()
            if wait > 0:
                time.sleep(wait)
            pending.append(pool.apply_async(_serve_ref_worker, (q,),
                                            callback=lambda r, i=i: done.__setitem__(i, (time.time(), r))))
        for a in pending:
            a.wait()
    fin = [done[i][0] - t0 for i in range(len(trace))]
    lat = [fin[i] - trace[i]["arrival"] for i in range(len(trace))]
    span = max(fin) - trace[0]["arrival"]
    value = len(trace) / span
    line = {"metric": SERVE_METRIC, "impl": "reference", "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": len(trace), "warmup": 0, "ms_per_step": 1e3 * span / len(trace), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "iterations_median": int(np.median([done[i][1][1] for i in range(len(trace))])),
            "config": dict(serve_config(args, 1), processes=P, host_cores=cores),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": P, "kind": "reference",
                             "sample": f"the full {len(trace)}-request trace submitted at its arrival times to {P} "
                                       f"single-threaded worker processes on {cores} host cores; latency = "
                                       f"completion - arrival on the wall clock"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _serve_ref_idle(_):
    sys.path.insert(0, ROOT)
    from oracle import ref
    return ref.available()


def run_serving(args, rank, world, local):
    import voluma_b200 as vb
    from voluma_b200 import cases
    trace = deal(serve_trace(args), rank, world)  # replicas: requests dealt round-robin to the ranks
    meshes = {}
    built = []
    for q in trace:
        if q["n"] not in meshes:
            meshes[q["n"]] = cases.lid_cavity(q["n"], 100.0)
        m, case = meshes[q["n"]]
        c = dict(case, nu=1.0 / q["Re"])
        built.append((q, m, c))
    modes = {}
    sampler = ClockSampler(local)
    for prec in ("mixed", "fp64"):
        s = vb.Server(device=local, hbm_budget=int(args.hbm_gb * (1 << 30)), max_active=args.max_active)
        # warm-up requests (untimed): contexts, graphs, first launches
        wm, wc = cases.lid_cavity(32, 100.0)
        for _ in range(args.warmup):
            s.submit(wm, wc, max_iter=50, residual_tol=1e-12)
        got = 0
        while got < args.warmup:
            got += len(s.collect(timeout=1.0))
        if prec == "mixed":
            sampler.start()
        t0 = s.clock() + 0.05
        for q, m, c in built:
            cc = dict(c)
            if prec == "mixed":
                cc = dict(c, p=dict(c["p"], precision="mixed"), pFinal=dict(c["pFinal"], precision="mixed"))
            s.submit(m, cc, arrival=t0 + q["arrival"], max_iter=20000, residual_tol=1e-6)
        res = []
        while len(res) < len(built):
            res += s.collect(timeout=1.0)
        if prec == "mixed":
            clocks = sampler.stop()
        s.close()
        ok = [r for r in res if r["status"] == 0]
        lat = [r["finished"] - r["arrival"] for r in ok]
        span = max(r["finished"] for r in ok) - min(r["arrival"] for r in ok)
        modes[prec] = dict(value=len(ok) / span, ms_per_step=1e3 * span / max(len(ok), 1),
                           p50_ms=1e3 * float(np.percentile(lat, 50)), p99_ms=1e3 * float(np.percentile(lat, 99)),
                           iterations_median=int(np.median([r["iterations"] for r in ok])),
                           failed=len(res) - len(ok), gpu_launches=int(sum(r["launches"] for r in ok)),
                           span_s=span)
    if world > 1:
        import torch
        span = max_over_ranks(modes["mixed"]["span_s"], world, torch.device("cuda", local))
        modes["mixed"]["value"] = args.requests / span
    if rank != 0:
        return
    mx = modes["mixed"]
    h2d = sum(8 * m["n_cells"] * 3 + 8 * 12 * m["n_faces"] for _, m, _ in built) // max(len(built), 1)
    d2h = sum(8 * (4 * m["n_cells"] + m["n_faces"]) for _, m, _ in built) // max(len(built), 1)
    line = {"metric": SERVE_METRIC, "value": mx["value"], "unit": "solves/s", "n_gpus": world,
            "steps": args.requests, "warmup": args.warmup, "ms_per_step": mx["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic",
            "p50_ms": mx["p50_ms"], "p99_ms": mx["p99_ms"], "config": serve_config(args, world),
            "modes": {"mixed": mx, "fp64": modes["fp64"],
                      "speedup_mixed_vs_fp64": modes["fp64"]["span_s"] / mx["span_s"]},
            "e2e": {"value": mx["value"], "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "note": "latency and throughput are end to end through vlm_server_* with host meshes: "
                            "registration (GAMG hierarchy), H2D, every SIMPLE step, D2H of U, p, phi"},
            "clocks": clocks, "gpu_launches": mx["gpu_launches"]}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ channel LES workload
CHAN_METRIC = "channel Re_tau 395 LES: PIMPLE steps/s (Smagorinsky + Van Driest, mean-velocity forcing)"
CHAN_REF_SAMPLE = (96, 72, 48)


def chan_shape(args):
    return tuple(int(v) for v in args.channel.split("x"))


def chan_config(args, world, n):
    return {"workload": f"periodic channel 2pi x 2 x pi, {n[0]}x{n[1]}x{n[2]} hex ({n[0] * n[1] * n[2]} cells), "
                        f"tanh wall grading (first cell y+ ~ 1 at Re_tau 395), nu = 1/6875 (Re_b 6875), "
                        f"mean-velocity forcing to Ubar = (1,0,0), Smagorinsky LES with Van Driest damping, "
                        f"PIMPLE backward/linear nOuter 1 nCorr 2, U PBiCGStab/DILU 1e-8, p PCG/GAMG 1e-8 "
                        f"(relTol 0.01, final 0); laminar profile + 10% seeded noise, dt at Courant ~0.5",
            "cells": n[0] * n[1] * n[2], "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (the 6.3M-cell step touches ~GBs)"}


def _chan_ref_step_time(n, steps):
    """Seconds per step of the reference's own LES channel step (IncompressibleFlow + TurbulenceModel,
    single-threaded) on an n-cell channel, excluding the first step."""
    sys.path.insert(0, ROOT)
    from oracle import ref
    from voluma_b200 import cases
    m, case, model, U0, dt = cases.channel(n)
    beta = cases.channel_beta(n[1], 1.0 / 395.0)
    R = ref.RefMesh(n, hi=(2 * np.pi, 2.0, np.pi), periodic=(1, 0, 1), beta=(0, beta, 0),
                    patch_types=[0, 0, 1, 1, 0, 0])
    t0 = time.perf_counter()
    R.flow_run(case, 1, dt=dt, U=U0, model=model)
    t1 = time.perf_counter()
    R.flow_run(case, 1 + steps, dt=dt, U=U0, model=model)
    t2 = time.perf_counter()
    return ((t2 - t1) - (t1 - t0)) / steps


def run_channel_reference(args, rank, world):
    """The reference's LES step timed on a bounded sample (a 96x72x48 channel, the same case), scaled to the
    configured channel by cells: steps/s = (cell-steps/s of the sample) / cells."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvlmref.so was not built (make -C oracle)"}))
        return
    n = chan_shape(args)
    cells = n[0] * n[1] * n[2]
    ns = CHAN_REF_SAMPLE
    per = _chan_ref_step_time(ns, 2)
    value = (ns[0] * ns[1] * ns[2] / per) / cells
    sample = f"2 LES channel steps on {ns[0]}x{ns[1]}x{ns[2]} cells (after one untimed step), 1 thread, scaled by cells"
    line = {"metric": CHAN_METRIC, "impl": "reference", "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": 2, "warmup": 1, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": chan_config(args, 1, n),
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_channel(args, rank, world, local):
    import torch
    import voluma_b200 as vb
    from voluma_b200 import cases
    torch.cuda.set_device(local)
    n = chan_shape(args)
    m, case0, model, U0, dt = cases.channel(n, seed=20261203 + rank)
    mesh = vb.Mesh.from_arrays(m, ctx=vb.Context(local))
    st = torch.cuda.ExternalStream(mesh.ctx.stream())
    modes = {}
    sampler = ClockSampler(local)
    clocks = None
    for prec in ("mixed", "fp64"):
        case = dict(case0, p=dict(case0["p"], precision=prec), pFinal=dict(case0["pFinal"], precision=prec))
        fl = vb.Flow(mesh, case)
        fl.set_model(model)
        fl.set_state(U0, None)
        for _ in range(args.warmup):
            fl.step(dt)
        l0 = fl.launches()
        if prec == "mixed":
            sampler.start()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its = 0
        for _ in range(args.steps):
            its += fl.step(dt)["iterations"]
        e1.record(st)
        torch.cuda.synchronize(local)
        dev_s = e0.elapsed_time(e1) / 1e3
        launches = fl.launches() - l0
        # end to end: every step also reads U and p back to the host
        t = time.perf_counter()
        for _ in range(max(2, args.steps // 2)):
            fl.step(dt)
            fl.state()
        e2e_s = max_over_ranks((time.perf_counter() - t) / max(2, args.steps // 2), world, torch.device("cuda", local))
        if prec == "mixed":
            clocks = sampler.stop()
        fl.close()
        dev_s = max_over_ranks(dev_s, world, torch.device("cuda", local))
        modes[prec] = dict(value=aggregate_rate(args.steps, world, dev_s), ms_per_step=1e3 * dev_s / args.steps,
                           iterations_per_step=its / args.steps, e2e_steps_per_s=world / e2e_s,
                           gpu_launches=int(launches))
    if rank != 0:
        return
    mx = modes["mixed"]
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            ns = CHAN_REF_SAMPLE
            per = _chan_ref_step_time(ns, 2)
            cpu = {"value": (ns[0] * ns[1] * ns[2] / per) / (n[0] * n[1] * n[2]), "unit": "steps/s", "cores": 1,
                   "kind": "reference",
                   "sample": f"2 LES channel steps on {ns[0]}x{ns[1]}x{ns[2]} cells, 1 thread, scaled by cells"}
    nC = n[0] * n[1] * n[2]
    line = {"metric": CHAN_METRIC, "value": mx["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (pressure V-cycle f32 in mixed)", "data": "synthetic",
            "config": chan_config(args, world, n),
            "modes": {"mixed": mx, "fp64": modes["fp64"],
                      "speedup_mixed_vs_fp64": modes["fp64"]["ms_per_step"] / mx["ms_per_step"]},
            "e2e": {"value": mx["e2e_steps_per_s"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * 4 * nC,
                    "note": "vlm_flow_step plus vlm_flow_get_state of U and p every step; the state stays resident"},
            "roofline": None, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": mx["gpu_launches"]}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ TGV PIMPLE workload (config 2)
TGV_METRIC = "Taylor-Green 3D PIMPLE: s/step (backward, dt 2e-3, nCorr 2, p PCG+GAMG 1e-8), FP64 vs mixed pressure"
TGV_DT = 2e-3


def tgv_config(args, world):
    return {"workload": f"3D Taylor-Green vortex, periodic box [0,2pi]^3, {args.n}^3 hex ({args.n ** 3} cells), nu = 1/1600, "
                        f"u0 = (sin x cos y cos z, -cos x sin y cos z, 0); transient PIMPLE backward, linear, dt = "
                        f"{TGV_DT}, nOuter 1, nCorr 2; U PBiCGStab/DILU 1e-8, p PCG/GAMG 1e-8 relTol 0.01, "
                        f"pFinal relTol 0", "cells": args.n ** 3, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (the step touches ~GBs)",
            "steps_note": "the configuration's 200 steps are not run: s/step is timed over the steps given"}


def _tgv_ref_step_time(n, steps):
    """Seconds per step of the reference's own PIMPLE step (IncompressibleFlow, single-threaded) on the
    n^3 TGV, over `steps` steps after one untimed step."""
    sys.path.insert(0, ROOT)
    from oracle import ref
    from voluma_b200 import cases
    m, case, U0 = cases.taylor_green_flow(n)
    R = ref.RefMesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    t0 = time.perf_counter()
    R.flow_run(case, 1, dt=TGV_DT, U=U0)
    t1 = time.perf_counter()
    _, _, _, hist = R.flow_run(case, 1 + steps, dt=TGV_DT, U=U0)
    t2 = time.perf_counter()
    return ((t2 - t1) - (t1 - t0)) / steps, float(np.mean(hist[1:, 3]))


def run_tgv_reference(args, rank, world):
    """The reference's own PIMPLE step on the same TGV, one process (its MPI path is not built here);
    s/step over 2 steps after an untimed one.  Higher is better is false: the metric is time."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvlmref.so was not built (make -C oracle)"}))
        return
    per, its = _tgv_ref_step_time(args.n, 2)
    line = {"metric": TGV_METRIC, "impl": "reference", "value": per, "unit": "s/step", "n_gpus": args.gpus,
            "steps": 2, "warmup": 1, "ms_per_step": 1e3 * per, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": tgv_config(args, 1),
            "linear_iterations_per_step": its,
            "cpu_baseline": {"value": per, "unit": "s/step", "cores": 1, "kind": "reference",
                             "sample": f"2 PIMPLE steps of the {args.n}^3 TGV after one untimed step, 1 thread "
                                       f"(reference IncompressibleFlow::step)"},
            "e2e": {"value": per, "unit": "s/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_tgv(args, rank, world, local):
    import torch
    import voluma_b200 as vb
    from voluma_b200 import cases
    torch.cuda.set_device(local)
    m, case0, U0 = cases.taylor_green_flow(args.n)
    mesh = vb.Mesh.from_arrays(m, ctx=vb.Context(local))
    st = torch.cuda.ExternalStream(mesh.ctx.stream())
    modes = {}
    sampler = ClockSampler(local)
    clocks = None
    fields = {}
    for prec in ("mixed", "fp64"):
        case = dict(case0, p=dict(case0["p"], precision=prec), pFinal=dict(case0["pFinal"], precision=prec))
        fl = vb.Flow(mesh, case)
        fl.set_state(U0, None)
        for _ in range(args.warmup):
            fl.step(TGV_DT)
        l0 = fl.launches()
        if prec == "mixed":
            sampler.start()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its = 0
        for _ in range(args.steps):
            its += fl.step(TGV_DT)["iterations"]
        e1.record(st)
        torch.cuda.synchronize(local)
        dev_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, world, torch.device("cuda", local))
        launches = fl.launches() - l0
        # end to end: every step also reads U and p back to the host
        t = time.perf_counter()
        ne = max(2, args.steps // 2)
        for _ in range(ne):
            fl.step(TGV_DT)
            U, p, _ = fl.state()
        e2e_s = max_over_ranks((time.perf_counter() - t) / ne, world, torch.device("cuda", local))
        if prec == "mixed":
            clocks = sampler.stop()
        fields[prec] = (U, p)
        fl.close()
        modes[prec] = dict(value=dev_s / args.steps, ms_per_step=1e3 * dev_s / args.steps,
                           linear_iterations_per_step=its / args.steps, e2e_s_per_step=e2e_s,
                           gpu_launches=int(launches))
    if rank != 0:
        return
    mx = modes["mixed"]
    u64, p64 = fields["fp64"]
    umx, pmx = fields["mixed"]
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            per, _ = _tgv_ref_step_time(min(args.n, 64), 2)
            scale = (args.n / min(args.n, 64)) ** 3
            cpu = {"value": per * scale, "unit": "s/step", "cores": 1, "kind": "reference",
                   "sample": f"2 PIMPLE steps of the {min(args.n, 64)}^3 TGV after one untimed step, 1 thread, "
                             f"scaled by cells to {args.n}^3"}
    line = {"metric": TGV_METRIC, "value": mx["value"], "unit": "s/step", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["ms_per_step"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (pressure V-cycle f32 in mixed)", "data": "synthetic",
            "config": tgv_config(args, world),
            "modes": {"mixed": mx, "fp64": modes["fp64"],
                      "speedup_mixed_vs_fp64": modes["fp64"]["ms_per_step"] / mx["ms_per_step"],
                      "extrapolated_200_steps_s": {"mixed": 200 * mx["value"], "fp64": 200 * modes["fp64"]["value"]},
                      "mixed_vs_fp64_after_steps": {
                          "U_rel_l2": float(np.linalg.norm(umx - u64) / np.linalg.norm(u64)),
                          "p_rel_l2": float(np.linalg.norm(pmx - p64) / np.linalg.norm(p64))}},
            "e2e": {"value": mx["e2e_s_per_step"], "unit": "s/step", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * 4 * args.n ** 3,
                    "note": "vlm_flow_step plus vlm_flow_get_state of U and p every step; the state stays resident"},
            "roofline": None, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": mx["gpu_launches"]}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ batch workload (config 3)
BATCH_METRIC = ("batch of Poisson systems: systems solved/s (laplacian with LS non-orthogonal correction, "
                "nNonOrthCorr 2, PCG+GAMG relTol 1e-8, FP32 V-cycles in FP64 PCG)")
BATCH_SEED = 20261203
BATCH_NON_ORTH = 2


def batch_params(args, rank=0):
    from voluma_b200 import cases
    return cases.poisson_batch_params(args.systems, 16, 96, seed=BATCH_SEED + rank, jitter=0.2, ratio_max=8.0)


def batch_config(args, world, cells):
    return {"workload": f"{args.systems} pressure Poisson systems (projectDivergenceFree): box meshes n^3, n uniform "
                        f"in [16, 96], tanh grading ratio U[1, 8], interior vertices jittered U(+-0.2h), Neumann "
                        f"walls + reference cell 0, RHS = div of 16 seeded Fourier modes (|k| <= 4, N(0,1)/|k|^2); "
                        f"laplacian(1, p) with least-squares non-orthogonal correction, nNonOrthCorr "
                        f"{BATCH_NON_ORTH}, PCG+GAMG relTol 1e-8 from p = 0; seed {BATCH_SEED}",
            "systems": args.systems, "cells": int(cells), "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (the batch holds ~1e8 cells)"}


def _batch_ref_worker(q):
    """One system through the reference's own pressure loop (laplacian + setReference + solveLdu,
    nNonOrthCorr + 1 passes), single-threaded: (seconds, cells)."""
    sys.path.insert(0, ROOT)
    from oracle import ref
    from voluma_b200 import cases
    from voluma_b200 import mesh as vm
    m, div = cases.poisson_system(q)
    n = q["n"]
    beta = math.acosh(math.sqrt(q["ratio"])) if q["ratio"] > 1.0 + 1e-12 else 0.0
    pts = vm.jitter_interior(vm.box_points((n, n, n), beta=(beta, beta, beta)), (n, n, n), q["jitter"], q["mesh_seed"])
    R = ref.RefMesh((n, n, n), beta=(beta, beta, beta), points=pts)
    t = time.perf_counter()
    R.pressure_solve(np.ones(m["n_faces"]), div, np.zeros(m["n_cells"]), ref_cell=0, n_non_orth=BATCH_NON_ORTH,
                     grad_scheme=1, rel_tol=1e-8, max_iter=1000)
    return time.perf_counter() - t, m["n_cells"]


def batch_reference_sample(args):
    """The reference on a bounded sample of the batch: its first `--ref-systems` systems, one
    single-threaded worker process per system (up to 16 concurrently); returns (systems/s at the
    batch's mean system size, cores, sample text)."""
    import multiprocessing as mp
    params = batch_params(args)
    sample = params[:args.ref_systems]
    P = max(1, min(os.cpu_count() or 1, 16, len(sample)))
    t = time.perf_counter()
    with mp.get_context("spawn").Pool(P) as pool:
        res = pool.map(_batch_ref_worker, sample, chunksize=1)
    wall = time.perf_counter() - t  # includes mesh generation in the workers: conservative
    solve_cells = sum(c for _, c in res)
    mean_cells = float(np.mean([q["n"] ** 3 for q in params]))
    busy = sum(d for d, _ in res)
    value = (solve_cells / busy) * P / mean_cells
    text = (f"the batch's first {len(sample)} systems ({solve_cells} cells), reference pressure loop per system in "
            f"{P} single-threaded processes; systems/s = cells solved per busy core-second x {P} cores / mean cells "
            f"per system of the full batch ({mean_cells:.0f}); wall {wall:.1f} s")
    return value, P, text


def run_batch_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libvlmref.so was not built (make -C oracle)"}))
        return
    value, P, text = batch_reference_sample(args)
    cells = sum(q["n"] ** 3 for q in batch_params(args))
    line = {"metric": BATCH_METRIC, "impl": "reference", "value": value, "unit": "systems/s", "n_gpus": args.gpus,
            "steps": args.ref_systems, "warmup": 0, "ms_per_step": 1e3 * args.systems / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": batch_config(args, 1, cells),
            "cpu_baseline": {"value": value, "unit": "systems/s", "cores": P, "kind": "reference", "sample": text},
            "e2e": {"value": value, "unit": "systems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_batch(args, rank, world, local):
    import torch
    from concurrent.futures import ThreadPoolExecutor
    import voluma_b200 as vb
    from voluma_b200 import cases
    params = batch_params(args, rank)
    keep = ("n_cells", "n_internal_faces", "n_faces", "owner", "neighbour", "magSf", "ndc", "V", "Sf", "d", "w",
            "corrVecs", "patch_start", "patch_size", "two_d", "empty_dir")

    def gen(q):  # only the arrays the registration reads: the batch's host copy stays ~half the size
        m, d = cases.poisson_system(q)
        return {k: m[k] for k in keep if k in m}, d
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        systems = list(ex.map(gen, params))
    t_gen = time.perf_counter() - t0
    meshes = [m for m, _ in systems]
    torch.cuda.set_device(local)
    ctx = vb.Context(local)
    t0 = time.perf_counter()
    B = vb.Mesh.batch(meshes, ctx=ctx)
    t_reg = time.perf_counter() - t0
    gamma_h = cases.batch_face_array(meshes, [np.ones(m["n_faces"]) for m in meshes])
    div_h = np.concatenate([d for _, d in systems])
    del systems
    dev = torch.device("cuda", local)
    st = torch.cuda.ExternalStream(ctx.stream())
    with torch.cuda.stream(st):
        gamma = torch.from_numpy(gamma_h).to(dev)
        div = torch.from_numpy(div_h).to(dev)
        p = torch.zeros(B.n_cells, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(local)
    refs = [0] * len(meshes)
    modes = {}
    sampler = ClockSampler(local)
    clocks = None
    for prec in ("mixed", "fp64"):
        ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000, precision="" if prec == "fp64" else prec)

        def one():
            with torch.cuda.stream(st):
                p.zero_()
            return vb.pressure_solve_device(B, gamma.data_ptr(), div.data_ptr(), p.data_ptr(), ctrl, ref_cell=refs,
                                            n_non_orth=BATCH_NON_ORTH, grad_scheme=1)
        for _ in range(args.warmup):
            perf = one()
        its = [[r.iterations for r in row] for row in perf]
        if prec == "mixed":
            sampler.start()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = B.stats()[0]
        e0.record(st)
        for _ in range(args.steps):
            perf = one()
        e1.record(st)
        torch.cuda.synchronize(local)
        launches = B.stats()[0] - l0
        dev_s = e0.elapsed_time(e1) / 1e3
        ok = all(r.converged for row in perf for r in row)
        if prec == "mixed":
            clocks = sampler.stop()
        dev_s = max_over_ranks(dev_s, world, dev)
        modes[prec] = dict(value=aggregate_rate(args.systems * args.steps, world, dev_s),
                           ms_per_step=1e3 * dev_s / args.steps, gpu_launches=int(launches),
                           all_converged=bool(ok), iterations_max=int(max(max(r) for r in its)),
                           iterations_median=int(np.median([x for r in its for x in r])))
    # plain FP64: every system registered on its own and solved one after another with the same
    # corrector (the unbatched FP64 GPU path), registration untimed
    if args.plain:
        singles = [vb.Mesh.from_arrays(mm, ctx=ctx) for mm in meshes]
        offs = np.cumsum([0] + [mm["n_cells"] for mm in meshes])
        with torch.cuda.stream(st):
            g1 = [torch.ones(mm["n_faces"], dtype=torch.float64, device=dev) for mm in meshes]
            p1 = [torch.zeros(mm["n_cells"], dtype=torch.float64, device=dev) for mm in meshes]
        ctrl64 = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000)

        def plain_pass():
            its = []
            for i, sm in enumerate(singles):
                with torch.cuda.stream(st):
                    p1[i].zero_()
                perf = vb.pressure_solve_device(sm, g1[i].data_ptr(), div.data_ptr() + 8 * int(offs[i]),
                                                p1[i].data_ptr(), ctrl64, ref_cell=0, n_non_orth=BATCH_NON_ORTH,
                                                grad_scheme=1)
                its.append(perf[-1][0].iterations)
            return its
        plain_pass()  # warm-up: every system's graphs
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its1 = plain_pass()
        e1.record(st)
        torch.cuda.synchronize(local)
        plain_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, world, dev)
        # the same systems' results as the batched FP64 solve
        with torch.cuda.stream(st):
            p.zero_()
        vb.pressure_solve_device(B, gamma.data_ptr(), div.data_ptr(), p.data_ptr(),
                                 vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000), ref_cell=refs,
                                 n_non_orth=BATCH_NON_ORTH, grad_scheme=1)
        torch.cuda.synchronize(local)
        pb = p.cpu().numpy()
        same = all(np.array_equal(p1[i].cpu().numpy(), pb[offs[i]:offs[i + 1]]) for i in range(len(singles)))
        modes["fp64_plain"] = dict(value=aggregate_rate(args.systems, world, plain_s), ms_per_step=1e3 * plain_s,
                                   iterations_median=int(np.median(its1)), iterations_max=int(max(its1)),
                                   bitwise_equal_to_batched_fp64=bool(same))
        del singles, g1, p1
    # end to end through the host-pointer corrector (H2D gamma, div, p; D2H p and the face flux)
    ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000, precision="mixed")
    ph = np.zeros(B.n_cells)
    t = time.perf_counter()
    ne = max(1, args.steps // 2)
    for _ in range(ne):
        ph[:] = 0.0
        vb.pressure_solve(B, gamma_h, div_h, ph, ctrl, ref_cell=refs, n_non_orth=BATCH_NON_ORTH, grad_scheme=1)
    e2e = aggregate_rate(args.systems * ne, world, max_over_ranks(time.perf_counter() - t, world, dev))
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            v, P, text = batch_reference_sample(args)
            cpu = {"value": v, "unit": "systems/s", "cores": P, "kind": "reference", "sample": text}
    mx = modes["mixed"]
    nC, nF = B.n_cells, B.n_faces
    line = {"metric": BATCH_METRIC, "value": mx["value"], "unit": "systems/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic",
            "config": batch_config(args, world, nC),
            "modes": dict({"mixed": mx, "fp64": modes["fp64"],
                           "speedup_mixed_vs_fp64": modes["fp64"]["ms_per_step"] / mx["ms_per_step"]},
                          **({"fp64_plain": modes["fp64_plain"],
                              "speedup_batched_mixed_vs_plain_fp64": modes["fp64_plain"]["ms_per_step"] /
                              mx["ms_per_step"]} if "fp64_plain" in modes else {})),
            "setup_s": {"generate": t_gen, "register": t_reg},
            "e2e": {"value": e2e, "unit": "systems/s", "h2d_bytes_per_step": int(8 * (nF + 2 * nC)),
                    "d2h_bytes_per_step": int(8 * (nC + nF)),
                    "note": "vlm_pressure_solve_batch with host arrays: H2D gamma, divPhi, p; D2H p and flux"},
            "roofline": None, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": modes["mixed"]["gpu_launches"]}
    print(json.dumps(line))


# ------------------------------------------------------------------------------ our arm
METRIC = "solves/s & p99 latency at rtol 1e-8, mixed vs FP64 GAMG-PCG on 1 B200"


def run_ours(args, rank, world, local):
    import torch
    import voluma_b200 as vb
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    m = our_mesh(args.n)
    diag, upper, b = assemble(m)
    n, nI = m["n_cells"], m["n_internal_faces"]
    ctx = vb.Context(local)
    mesh = vb.Mesh.from_arrays(m, ctx=ctx)
    ext = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    d_diag = torch.from_numpy(diag).to(dev)
    d_up = torch.from_numpy(upper).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.zeros(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def ctrl(prec):
        return vb.SolverControls("PCG", "GAMG", 0.0, REL_TOL, 1000, smoother=args.smoother,
                                 precision={"mixed": "mixed", "mixed_dc": "mixed-dc"}.get(prec, ""))

    def device_solve(prec, on=None):
        with torch.cuda.stream(ext):
            d_x.zero_()
        return vb.solve_ldu_device(on or mesh, d_diag.data_ptr(), d_up.data_ptr(), 0, d_b.data_ptr(), d_x.data_ptr(),
                                   ctrl(prec))

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    modes = {}
    sampler = ClockSampler(local)
    for prec in ("fp64", "mixed"):
        for _ in range(args.warmup):
            device_solve(prec)
        barrier()
        if prec == "mixed":
            sampler.start()
        l0 = mesh.stats()[0]
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        perfs = []
        for e0, e1 in ev:
            with torch.cuda.stream(ext):
                d_x.zero_()
            e0.record(ext)
            perfs.append(vb.solve_ldu_device(mesh, d_diag.data_ptr(), d_up.data_ptr(), 0, d_b.data_ptr(),
                                             d_x.data_ptr(), ctrl(prec)))
            e1.record(ext)
        barrier()
        launches = mesh.stats()[0] - l0
        ms = np.array([e0.elapsed_time(e1) for e0, e1 in ev])
        tot = float(ms.sum())
        tot = max_over_ranks(tot, world, dev)
        modes[prec] = dict(value=aggregate_rate(args.steps, world, tot / 1e3), ms_per_step=tot / args.steps,
                           p50_ms=float(np.percentile(ms, 50)), p99_ms=float(np.percentile(ms, 99)),
                           iterations=int(np.median([p.iterations for p in perfs])),
                           outer=int(np.median([p.outerIterations for p in perfs])),
                           final_rel=float(max(p.finalResidual / max(p.initialResidual, 1e-300) for p in perfs)),
                           converged=all(p.converged for p in perfs), gpu_launches=int(launches))
    clocks = sampler.stop()
    x_mixed = d_x.cpu().numpy()
    device_solve("fp64")
    x64 = d_x.cpu().numpy()
    err_vs_fp64 = float(np.linalg.norm(x_mixed - x64) / np.linalg.norm(x64))

    # FP64 defect correction around an FP32 inner PCG (the reference mode projected out), beside
    for _ in range(args.warmup):
        device_solve("mixed_dc")
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    perfs = []
    for e0, e1 in ev:
        with torch.cuda.stream(ext):
            d_x.zero_()
        e0.record(ext)
        perfs.append(vb.solve_ldu_device(mesh, d_diag.data_ptr(), d_up.data_ptr(), 0, d_b.data_ptr(),
                                         d_x.data_ptr(), ctrl("mixed_dc")))
        e1.record(ext)
    barrier()
    tot = max_over_ranks(float(sum(e0.elapsed_time(e1) for e0, e1 in ev)), world, dev)
    x_dc = d_x.cpu().numpy()
    modes["mixed_dc"] = dict(value=aggregate_rate(args.steps, world, tot / 1e3), ms_per_step=tot / args.steps,
                             iterations=int(np.median([p.iterations for p in perfs])),
                             outer=int(np.median([p.outerIterations for p in perfs])),
                             final_rel=float(max(p.finalResidual / max(p.initialResidual, 1e-300) for p in perfs)),
                             converged=all(p.converged for p in perfs),
                             rel_l2_vs_fp64=float(np.linalg.norm(x_dc - x64) / np.linalg.norm(x64)))

    # the same solves on the device-built hierarchy (parallel matching, vlm_mesh_register_ex):
    # registration time and the solve rates beside the reference hierarchy's
    barrier()
    t_reg = time.perf_counter()
    mesh_dev = vb.Mesh.from_arrays(m, ctx=ctx, agglomeration="device")
    t_reg = time.perf_counter() - t_reg
    dev_modes = {"registration_s": t_reg}
    for prec in ("fp64", "mixed"):
        for _ in range(args.warmup):
            device_solve(prec, mesh_dev)
        barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        perfs = []
        for e0, e1 in ev:
            with torch.cuda.stream(ext):
                d_x.zero_()
            e0.record(ext)
            perfs.append(vb.solve_ldu_device(mesh_dev, d_diag.data_ptr(), d_up.data_ptr(), 0, d_b.data_ptr(),
                                             d_x.data_ptr(), ctrl(prec)))
            e1.record(ext)
        barrier()
        tot = max_over_ranks(float(sum(e0.elapsed_time(e1) for e0, e1 in ev)), world, dev)
        dev_modes[prec] = dict(value=aggregate_rate(args.steps, world, tot / 1e3), ms_per_step=tot / args.steps,
                               iterations=int(np.median([p.iterations for p in perfs])),
                               converged=all(p.converged for p in perfs))
    mesh_dev.close()

    # e2e: host pinned buffers through vlm_ldu_solve (H2D diag/upper/b/x, D2H x inside the timed region)
    h_diag = torch.from_numpy(diag).pin_memory().numpy()
    h_up = torch.from_numpy(upper).pin_memory().numpy()
    h_b = torch.from_numpy(b).pin_memory().numpy()
    h_x = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        h_x[:] = 0.0
        vb.solve_ldu(mesh, h_diag, h_up, None, h_b, h_x, ctrl("mixed"))
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        h_x[:] = 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        vb.solve_ldu(mesh, h_diag, h_up, None, h_b, h_x, ctrl("mixed"))
        e1.record(ext)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    e2e_tot = max_over_ranks(float(np.sum(e2e_ms)), world, dev)

    # roofline of the dominant kernel (level-0 red-black GS sweep of the FP32 inner V-cycle), timed
    # with CUDA events on the context stream inside one mixed solve: an event pair around every
    # level-0 sweep, launches in the solve's own order (so each sweep meets the cache state the
    # V-cycle leaves it).  Beside it: the sweep alone after an L2-evicting 256 MB read (cold), back
    # to back (warm: its 59 MB of operands stay in L2) and as two colour launches.
    h_x[:] = 0.0
    mesh.time_sweeps(True)
    vb.solve_ldu(mesh, h_diag, h_up, None, h_b, h_x, ctrl("mixed"))
    sweep_ms, sweeps = mesh.sweep_time()
    mesh.time_sweeps(False)
    k_ms = sweep_ms / max(sweeps, 1)
    k_ms_cold, k_bytes = mesh.profile_kernel("smooth32", 20)
    k_ms_warm, _ = mesh.profile_kernel("smooth32:warm", 20)
    k_ms_steps, _ = mesh.profile_kernel("smooth32_steps", 20)
    # the FP64 Krylov product of the same system (plane-streamed where the mesh allows it)
    p_ms_cold, p_bytes = mesh.profile_kernel("spmv64", 20)
    p_ms_warm, _ = mesh.profile_kernel("spmv64:warm", 20)
    streamed = mesh.stream_config()[2] > 0
    peak, peak_kind = measured_peak_gbs()
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic = ncu_traffic("smooth32", args.n)
    if rank != 0:
        return
    mx = modes["mixed"]
    line = {
        "metric": METRIC, "value": mx["value"], "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mx["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic",
        "p50_ms": mx["p50_ms"], "p99_ms": mx["p99_ms"],
        "config": pressure_config(args.n, world, args.smoother),
        "modes": {"mixed": mx, "fp64": modes["fp64"],
                  "speedup_mixed_vs_fp64": modes["fp64"]["ms_per_step"] / mx["ms_per_step"],
                  "mixed_rel_l2_vs_fp64": err_vs_fp64,
                  "mixed_dc": modes["mixed_dc"],
                  "device_agglomeration": dev_modes},
        "e2e": {"value": world * args.steps / (e2e_tot / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": int(8 * (n + nI + n + n)), "d2h_bytes_per_step": int(8 * n),
                "p99_ms": float(np.percentile(e2e_ms, 99))},
        "fp64_product": {"kernel": ("k_box_pcg_spmv_stream<double>" if streamed else "k_box_pcg_spmv4<double>") +
                                    " level 0 (PCG product Ap = A p with the fused p.Ap)",
                         "alg_bytes_per_launch": p_bytes, "ms_per_launch_l2_cold": p_ms_cold,
                         "ms_per_launch_l2_warm": p_ms_warm, "peak": peak, "unit": "GB/s",
                         "frac_cold": p_bytes / (p_ms_cold * 1e-3) / 1e9 / peak,
                         "frac_warm": p_bytes / (p_ms_warm * 1e-3) / 1e9 / peak,
                         "timing": "CUDA events around single launches after an L2-evicting 256 MB read (cold) "
                                   "and around back-to-back launches (warm)"},
        "roofline": {"kernel": ("k_box_sweep4<float> level 0 (one full red-black Gauss-Seidel sweep, one launch)"
                                if os.environ.get("VLM_BOX_FUSED") == "1" else
                                "k_box_gs4<float> level 0 (one full red-black Gauss-Seidel sweep: two colour launches)"),
                     "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "ms_per_launch": k_ms,
                     "alg_bytes_per_launch": k_bytes,
                     "timing": f"live: mean of the {sweeps} level-0 sweeps of one mixed solve, CUDA events "
                               "around each sweep in the solve's launch order",
                     "ms_per_launch_l2_cold": k_ms_cold, "ms_per_launch_l2_warm": k_ms_warm,
                     "ms_per_sweep_as_two_colour_launches": k_ms_steps},
        "clocks": clocks, "gpu_launches": mx["gpu_launches"],
        "launch_configuration": launch_configuration(mesh),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n, diag, upper, b)
    print(json.dumps(line))


def launch_configuration(mesh):
    """The V-cycle launch shape the mesh ran with: coarse tail (from the tuner's table, or the
    built-in default with VLM_TUNE=0) and the fusion row limits."""
    from voluma_b200 import tune
    cl, max_rows, full_rows = mesh.tail_config()
    entry = tune.lookup(tune.load_table(mesh.ctx.device_name()), int(mesh.n_cells), 1) \
        if os.environ.get("VLM_TUNE", "1") != "0" else None
    return {"tail_cluster": cl, "tail_max_rows": max_rows, "tail_full_rows": full_rows,
            "tuning_entry": entry["case"] if entry else None,
            "tuning_table": os.path.relpath(tune.table_path(mesh.ctx.device_name()), ROOT) if entry else None,
            "fusion_rows": list(mesh.fusion_config())}


def cpu_baseline(n, diag, upper, b):
    """One reference solve of the same system on one host core (oracle/_ref), else the port."""
    try:
        from oracle import ref
        if ref.available():
            R = ref.RefMesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
            R.gamg_levels()
            t = time.perf_counter()
            _, perf = R.solve(diag, upper, None, b, np.zeros(R.n_cells), "PCG", "GAMG", 0.0, REL_TOL, 1000)
            dt = time.perf_counter() - t
            return {"value": 1.0 / dt, "unit": "solves/s", "cores": 1, "kind": "reference",
                    "sample": f"one full PCG+GAMG solve of the same {n}^3 system by the reference's solveLdu "
                              f"({perf['iterations']} iterations, {dt:.1f} s; hierarchy pre-built as the "
                              f"reference caches it on the Mesh)"}
    except Exception as e:  # pragma: no cover
        return {"value": None, "unit": "solves/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}
    return {"value": None, "unit": "solves/s", "cores": 1, "kind": "reference", "sample": "reference not built"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--smoother", default="")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="pressure", choices=["pressure", "serving", "channel", "batch", "tgv"])
    ap.add_argument("--systems", type=int, default=256)
    ap.add_argument("--ref-systems", type=int, default=16)
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="batch workload: skip the unbatched FP64 arm (each system solved on its own)")
    ap.add_argument("--channel", default="256x192x128")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--nmin", type=int, default=32)
    ap.add_argument("--nmax", type=int, default=256)
    ap.add_argument("--remin", type=float, default=100.0)
    ap.add_argument("--remax", type=float, default=1000.0)
    ap.add_argument("--max-active", type=int, default=8)
    ap.add_argument("--hbm-gb", type=float, default=64.0)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        {"serving": run_serving_reference, "channel": run_channel_reference,
         "batch": run_batch_reference, "tgv": run_tgv_reference}.get(args.workload, run_reference)(
            args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        {"serving": run_serving, "channel": run_channel, "batch": run_batch, "tgv": run_tgv}.get(args.workload, run_ours)(
            args, rank, world, local)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
