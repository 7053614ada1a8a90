#!/usr/bin/env python3
"""Benchmark of the RK3W fractional-step hot path on B200.

Default workload: the turbulent-channel configuration (96 x 64 x 64 hex cells, tanh-stretched,
KEP advection, Vreman SGS, log-law wall model, constant pressure-gradient forcing), synthetic
inputs (seeded laminar-plus-noise initial state).  One "step" is one RK3W time step (three
stages, three Poisson solves) of the whole mesh.  The timed form is the chosen pressure solve
(flexible CG with the two-level preconditioner on this mesh, the multilevel one on meshes too
large for it; both with the learned term trained and gated); on one GPU the plain FP64
Jacobi-PCG form is timed beside it on the same workload and reported in the config.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--config channel|channel3m|tgv|rb|mixed|urban] [--psolver auto|fcg|pcg|ml] [--no-plain]

(--psolver auto, the default, takes the two-level form when the mesh fits it — up to 4096 cells
per SM — and the multilevel form otherwise, as for the rb, mixed and urban configurations)

value   : cell-steps/s with the state resident in HBM (CUDA events around K steps, max over ranks)
e2e     : the same metric through the C ABI with host buffers: every step uploads the state
          (U, p) from pinned host memory, advances, and reads the state back
roofline: the Poisson kernel (dominant): algorithmic bytes per launch / average launch time
cpu_baseline: the CPU restatement of the reference step (oracle) on this host's cores, on a
          bounded sample of the same workload.
Multi-GPU: the north-star path is single-GPU; N GPUs run N independent replicas (weak scaling).
"""
import argparse
import ctypes as C
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

METRIC = "cell-steps/s & Poisson ms/step, learned+mixed vs plain FP64 PCG, 1 B200"


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def start(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.samples)}
        if self.samples:
            sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
            mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
            out["sm_mhz"] = statistics.median(sm) if sm else None
            out["sm_max_mhz"] = max(mx) if mx else None
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = set()
            for s in self.samples:
                for k, nm in enumerate(names):
                    if s[5 + k].lower() == "active":
                        reasons.add(nm)
            out["reasons"] = sorted(reasons)
        return out


FORMS = {"pcg": "plain FP64 Jacobi-PCG",
         "fcg": "FP64 flexible CG, deflated two-level preconditioner (148 parts, FP32 part-local Chebyshev "
                "degree 7 in shared memory + one coarse value per part)"}


FORMS["ml"] = ("FP64 flexible CG preconditioned by one FP32 aggregation-multigrid V-cycle (pairwise "
               "aggregation, 3 passes per level, Chebyshev degree 3, dense coarsest level)")
KERNELS = {"pcg": "k_pcg (persistent Jacobi-PCG)", "fcg": "k_fcg (persistent two-level flexible CG)",
           "ml": "k_mlcg (persistent multilevel flexible CG)"}


def make_case(name):
    from dopamine_b200 import cases
    if name == "channel":
        return cases.channel_config(96, 64, 64)
    if name == "tgv":
        return cases.tgv_config(64)
    if name == "channel3m":
        return cases.channel_config(192, 128, 128)
    if name == "rb":
        return cases.rb_config(256, 256, 128)
    if name == "mixed":
        return cases.hybrid_config(n=128, kind="mixed")
    if name == "urban":
        return cases.urban_config()
    raise ValueError(name)


def pcg_bytes_per_iteration(s, psolver="pcg"):
    """Algorithmic bytes of one Krylov iteration, per the ELL operator width (hex: 7)."""
    nc = s.nc
    wa = 7  # hex mesh: diagonal + 6 neighbours
    if psolver == "ml":
        # fine level only (the coarser levels add about 1/7): 2k = 6 FP32 smoothing/restriction
        # passes (cols + FP32 vals, b, d in/out, x in/out), the FP64 w = A z pass (cols, vals, z,
        # r, q in, w out) and the update pass (z, w, p, q, x, r in; p, q, x, r out; b, d, x0 out)
        k = 3
        return nc * (2 * k * (wa * (4 + 4) + 16) + (wa * (4 + 8) + 4 + 8 + 16) + (12 + 32 + 32 + 12))
    if psolver == "fcg":
        # w = A z: cols + vals, z gathered once per cell, z written once; the part-local smoother
        # and the own-cell vectors live in shared memory and registers
        # plus the deflation data (row sum, cross-coupling offsets) of the own rows
        return nc * (wa * (4 + 8) + 8 + 8 + 8)
    phase_a = nc * (wa * (4 + 8) + 8 + 8 + 8 + 8)   # cols, vals, z, p_old, write p_new, write q
    phase_b = nc * (5 * 8 + 3 * 8)                  # x, p, r, q, dinv in; x, r, z out
    return phase_a + phase_b


def pcg_traffic_per_launch(psolver="pcg"):
    """DRAM bytes (read + write) of one launch of the Poisson kernel on this workload, from the
    committed ncu summary (one capture, its command inside the file); None when absent."""
    name = {"fcg": "k_fcg_channel96x64x64.md", "ml": "k_mlcg_channel96x64x64.md"}.get(psolver, "k_pcg_channel96x64x64.md")
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


def max_over_ranks(values, device):
    """Element-wise maximum of per-rank timings over the process group (replicas: the job is as
    slow as its slowest rank)."""
    import torch
    t = torch.tensor(values, device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t]


def whole_job_rate(world, cells, steps, seconds):
    """cell-steps/s of N replicas that each advance `cells` cells `steps` times in `seconds`."""
    return world * cells * steps / seconds


def run_gpu(args, rank, world):
    import torch
    from dopamine_b200.solver import Solver, lib

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    case = make_case(args.config)
    if args.psolver == "auto":
        case.params["p_solver"] = 3  # DPM_PSOLVER_AUTO: two-level when the mesh fits it, else multilevel
    if args.psolver == "ml":
        case.params["p_solver"] = 2  # DPM_PSOLVER_MULTILEVEL_FCG
    if args.psolver == "fcg":
        case.params["p_solver"] = 1  # DPM_PSOLVER_TWOLEVEL_FCG
    if args.mixed and args.psolver in ("fcg", "auto"):
        case.params["form"] = 1  # DPM_FORM_MIXED (the multilevel form's V-cycle is FP32 already)
    s = Solver(case, device=dev)
    s.initialise()
    nc = s.nc
    learn = None
    if args.psolver == "auto":  # report the form the solver chose
        args.psolver = {0: "pcg", 1: "fcg", 2: "ml"}[s.stats()["p_solver_used"]]
    if args.psolver in ("fcg", "ml") and not args.no_learned:
        # learned preconditioner term: samples from 3 steps' solves, 80 Adam steps, gamma set on the
        # held-out solve (set-up work, outside the timed region; reported in the config)
        n_samples = s.learn_collect(3)
        learn = s.learn_train(epochs=80, lr=1e-2)
        learn["collect_steps"] = 3
        learn["samples_recorded"] = n_samples
    for _ in range(args.warmup):
        s.advance()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
    l0 = s.kernel_launches()
    step_ms, pois_ms, its, solves = [], [], 0, 0
    for _ in range(args.steps):
        s.advance()
        st = s.stats()
        a, b = s.last_timing()
        step_ms.append(a)
        pois_ms.append(b)
        its += st["p_iters"]
        solves += st["p_solves"]
    launches = s.kernel_launches() - l0
    t_dev = sum(step_ms) / 1e3
    # ---- end to end through the C ABI with host buffers
    L = lib()
    host = s.sync_host()
    # pinned host buffers (page-locked through torch), filled with the current state
    U_pin = torch.empty(host["U"].shape, dtype=torch.float64, pin_memory=True)
    p_pin = torch.empty(host["p"].shape, dtype=torch.float64, pin_memory=True)
    U = U_pin.numpy()
    p = p_pin.numpy()
    U[...] = host["U"]
    p[...] = host["p"]
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = L.dpm_upload_state(s.h, dp(U), dp(p), None)
        rc |= L.dpm_advance(s.h, s.params.dt)
        rc |= L.dpm_download_state(s.h, dp(U), dp(p), None, None)
        if rc:
            raise RuntimeError(f"e2e step failed {rc}")
    t_e2e = time.perf_counter() - t0
    clocks = sampler.stop() if sampler else None
    if world > 1:
        t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], "cuda")
    return dict(nc=nc, t_dev=t_dev, t_e2e=t_e2e, step_ms=step_ms, pois_ms=pois_ms, its=its, solves=solves,
                launches=launches, clocks=clocks, solver=s, learn=learn, fallbacks=s.stats()["p_fallbacks"])


def time_plain(args, dev, steps=3):
    """The plain FP64 Jacobi-PCG form on the same workload: device ms per step and Poisson ms
    per step (CUDA events inside the library), after one warm-up step."""
    from dopamine_b200.solver import Solver
    case = make_case(args.config)
    case.params["p_solver"] = 0
    s = Solver(case, device=dev)
    s.initialise()
    s.advance()
    step_ms, pois_ms, its = [], [], 0
    for _ in range(steps):
        s.advance()
        a, b = s.last_timing()
        step_ms.append(a)
        pois_ms.append(b)
        its += s.stats()["p_iters"]
    s.close()
    return sum(step_ms) / steps, sum(pois_ms) / steps, its / steps


def cpu_baseline(case_name, budget_s=20.0, nthreads=None):
    """The oracle (CPU restatement of the reference step) on this host, bounded sample."""
    from oracle.oracle import Oracle
    nthreads = nthreads or os.cpu_count() or 1
    case = make_case(case_name)
    o = Oracle(case, nthreads=nthreads)
    o.initialise()
    t0 = time.perf_counter()
    steps = 0
    while True:
        o.advance()
        steps += 1
        if time.perf_counter() - t0 >= budget_s or steps >= 3:
            break
    dt = time.perf_counter() - t0
    return dict(value=o.nc * steps / dt, unit="cell-steps/s", cores=nthreads, kind="port",
                sample=f"{steps} RK3W step(s) of the {case_name} workload ({o.nc} cells) after the initial projection, "
                       f"{dt:.1f} s, oracle with {nthreads} OpenMP threads")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dopamine_b200")
    ap.add_argument("--config", default="channel", choices=["channel", "channel3m", "tgv", "rb", "mixed", "urban"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 Jacobi-PCG form")
    ap.add_argument("--no-learned", action="store_true", help="flexible CG without the learned term")
    ap.add_argument("--mixed", action="store_true",
                    help="precision form: FP32-operator inner iterations inside FP64 defect correction")
    ap.add_argument("--psolver", default="auto", choices=["auto", "pcg", "fcg", "ml"],
                    help="auto: fcg when the mesh fits the two-level kernel, else ml; pcg: plain FP64 "
                         "Jacobi-PCG; fcg: flexible CG, two-level part-local preconditioner; "
                         "ml: flexible CG, aggregation-multigrid V-cycle")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    cfg_name = {"channel": "channel 96x64x64 Re_tau=395, KEP, Vreman, log-law wall model",
                "tgv": "Taylor-Green 64^3, CDS",
                "channel3m": "channel 192x128x128 (3.1M cells) Re_tau=395, KEP, Vreman, log-law wall model",
                "rb": "Rayleigh-Benard 256x256x128 (8.4M cells), Ra=1e7, Pr=0.7, T + 2 scalars van Leer, Vreman",
                "mixed": "jittered unit box 128^3 as hexes + prisms + pyramids (4.9M cells), AMD, Koren TVD",
                "urban": "urban canopy 1000x1000x300 m, 400x400x125 with 200 seeded obstacles carved out "
                         "(19.3M cells), MOST (L = -100 m), AMD, KEP, T + 1 scalar"}[args.config]

    if args.impl == "reference":
        if rank != 0:
            return 0
        cb = cpu_baseline(args.config, budget_s=60.0)
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg_name, "form": "plain FP64 Jacobi-PCG (CPU restatement)"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0

    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    r = run_gpu(args, rank, world)
    s = r["solver"]
    if world > 1:
        import torch
        torch.distributed.barrier()
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    nc, K = r["nc"], args.steps
    value = whole_job_rate(world, nc, K, r["t_dev"])
    e2e = whole_job_rate(world, nc, K, r["t_e2e"])
    peak, peak_kind = measured_peaks()
    bytes_it = pcg_bytes_per_iteration(s, args.psolver)
    pois_s = sum(r["pois_ms"]) / 1e3
    achieved = bytes_it * r["its"] / pois_s / 1e9 if pois_s > 0 else 0.0
    traffic = pcg_traffic_per_launch(args.psolver) if args.config == "channel" else None
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": 1e3 * r["t_dev"] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": cfg_name, "cells": nc, "form": FORMS[args.psolver],
                   "poisson_ms_per_step": 1e3 * pois_s / K, "pcg_iterations_per_step": r["its"] / K,
                   "poisson_solves_per_step": r["solves"] / K,
                   "l2": "inputs larger than L2: static operator data streamed each step exceeds 126 MB",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": 32 * nc, "d2h_bytes_per_step": 32 * nc},
        "roofline": {"kernel": KERNELS[args.psolver], "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "bytes_per_iteration": bytes_it},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    if args.mixed and args.psolver == "fcg":
        line["config"]["form"] += "; precision form (FP32-operator inner iterations, FP64 defect correction)"
    if r["learn"] is not None:
        line["config"]["learned_term"] = r["learn"]
        line["config"]["form"] += "; learned one-ring term (gamma %g)" % r["learn"]["gamma"]
    if args.psolver in ("fcg", "ml"):
        line["config"]["fallbacks_to_plain_pcg"] = r["fallbacks"]
    if args.psolver != "pcg" and not args.no_plain and world == 1:
        pm, pp, pit = time_plain(args, int(os.environ.get("LOCAL_RANK", "0")))
        line["config"]["plain_fp64_pcg"] = {"ms_per_step": pm, "poisson_ms_per_step": pp,
                                            "pcg_iterations_per_step": pit,
                                            "speedup_of_this_form": pm / line["ms_per_step"]}
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline is reported at N = 1 only
        cb = cpu_baseline(args.config, budget_s=20.0)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line))
    s.close()
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
