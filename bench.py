#!/usr/bin/env python3
"""Benchmark of the RK3W fractional-step hot path on B200.

Default workload: the urban-canopy configuration named by the metric ("learned+mixed vs plain
FP64 PCG"): a 1000 x 1000 x 300 m box at 400 x 400 x 125 hexes with 200 seeded cuboid obstacles
carved out (19.3 M cells), MOST wall model (L = -100 m), AMD SGS, KEP momentum, temperature plus
one passive scalar (van Leer), synthetic inputs (seeded uniform flow with +-10 % noise).  One
"step" is one RK3W time step (three stages, three Poisson solves) of the whole mesh.  The timed
form is the chosen pressure solve (flexible CG with the two-level preconditioner when the mesh
fits it, else with the FP32 aggregation-multigrid V-cycle; the learned term trained on 3
recorded steps and gated on a held-out solve) in the precision form (FP32 explicit half: first
gradient pass, SGS and flux assembly; FP64 state and projection; `--fp64` for the FP64 explicit
half); on one GPU the plain FP64 Jacobi-PCG form is timed beside it on the same handle, mesh and
state and reported in the config.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--fp64]
                    [--config urban|channel|channel3m|tgv|rb|mixed] [--psolver auto|fcg|pcg|ml] [--no-plain]

value   : cell-steps/s with the state resident in HBM (CUDA events around K steps, max over ranks)
e2e     : the same metric through the C ABI with host buffers: every step uploads the transported
          state (U, p, and T and the scalars when present) from pinned host memory, advances, and
          reads it back
roofline: the Poisson kernel (dominant): algorithmic bytes per launch / average launch time
cpu_baseline: the CPU restatement of the reference step (oracle) on this host's cores, on a
          bounded sample of the same workload (the sample is stated in the line).
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


FORMS["ml"] = ("FP64 flexible CG preconditioned by one aggregation-multigrid V-cycle on D^-1-scaled FP32 levels "
               "(pairwise aggregation, 3 passes per level, dense coarsest level; meshes of >= 2^20 cells: "
               "standalone full-occupancy kernels, Chebyshev degree 2; smaller: one persistent kernel, degree 3)")
KERNELS = {"pcg": "k_pcg (persistent Jacobi-PCG)", "fcg": "k_fcg (persistent two-level flexible CG)",
           "ml": "multilevel flexible CG (k_mlk_* standalone kernels on >= 2^20 cells, else persistent k_mlcg): "
                 "whole pressure solve"}


CONFIG_NAMES = {
    "urban": "urban canopy 1000x1000x300 m, 400x400x125 hexes with 200 seeded obstacles carved out (19.3M cells), "
             "MOST (L = -100 m), AMD, KEP, T + 1 scalar van Leer",
    "urban2m": "urban canopy 1000x1000x300 m at half resolution, 200x200x63 hexes with the same 200 obstacles "
               "(2.4M cells), MOST (L = -100 m), AMD, KEP, T + 1 scalar van Leer",
    "channel": "channel 96x64x64 Re_tau=395, KEP, Vreman, log-law wall model",
    "tgv": "Taylor-Green 64^3, CDS",
    "channel3m": "channel 192x128x128 (3.1M cells) Re_tau=395, KEP, Vreman, log-law wall model",
    "rb": "Rayleigh-Benard 256x256x128 (8.4M cells), Ra=1e7, Pr=0.7, T + 2 scalars van Leer, Vreman",
    "mixed": "jittered unit box 128^3 as hexes + prisms + pyramids (4.9M cells), AMD, Koren TVD",
}

# What stays in the 126 MB L2 and what streams from HBM, per workload (said in the line's config)
L2_NOTE = {
    "urban": "inputs larger than L2: the fine-level operator and vectors alone are ~1.5 GB; no flush needed",
    "urban2m": "inputs larger than L2: the fine-level operator and vectors alone are ~0.2 GB; no flush needed",
    "rb": "inputs larger than L2: the fine-level operator and vectors alone are ~0.7 GB; no flush needed",
    "mixed": "inputs larger than L2: the fine-level operator and vectors alone are ~0.5 GB; no flush needed",
    "channel3m": "inputs larger than L2: the fine-level operator and vectors alone are ~0.3 GB; no flush needed",
    "channel": "step data larger than L2 (LS weights alone 245 MB, streamed each gradient pass); the Poisson "
               "working set (operator 33 MB + vectors) is L2-resident, as the channel profiles show",
    "tgv": "step data larger than L2 (LS weights 1.6 GB); the Poisson working set is partly L2-resident",
}


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
    if name == "urban2m":
        return cases.urban_config(200, 200, 63)
    raise ValueError(name)


def cpu_sample_case(name):
    """The bounded CPU sample of a workload: the workload itself when the oracle steps it in
    seconds, else the same generator at reduced resolution.  Jacobi-PCG iterations per solve grow
    with the mesh's linear size, so a reduced mesh's CPU rate is an upper bound on the CPU's rate
    at full size (the GPU/CPU ratio is understated, not inflated)."""
    from dopamine_b200 import cases
    if name == "urban":
        return (cases.urban_config(100, 100, 32),
                "the urban generator at 1/4 linear resolution (100x100x32 hexes, same 1000x1000x300 m domain, "
                "the same 200 obstacles, 0.31M cells); Jacobi-PCG there needs ~1/3 of the full mesh's iterations "
                "per cell, so this rate is an upper bound on the CPU's full-size rate")
    if name == "urban2m":
        return (cases.urban_config(100, 100, 32),
                "the urban generator at 1/4 of the full linear resolution (100x100x32, 0.31M cells)")
    if name == "rb":
        return (cases.rb_config(64, 64, 32), "the Rayleigh-Benard generator at 1/4 linear resolution (64x64x32)")
    if name == "mixed":
        return (cases.hybrid_config(n=32, kind="mixed"), "the mixed-element generator at 1/4 linear resolution (n=32)")
    if name == "channel3m":
        return (cases.channel_config(96, 64, 64), "the channel generator at 1/2 linear resolution (96x64x64)")
    return make_case(name), f"the {name} workload itself"


def host_cores():
    """(threads this process may use, physical cores of the host)."""
    try:
        threads = len(os.sched_getaffinity(0))
    except AttributeError:
        threads = os.cpu_count() or 1
    phys = set()
    try:
        pid = cid = None
        for line in open("/proc/cpuinfo"):
            if line.startswith("physical id"):
                pid = line.split(":")[1].strip()
            elif line.startswith("core id"):
                cid = line.split(":")[1].strip()
            elif not line.strip():
                if cid is not None:
                    phys.add((pid, cid))
                pid = cid = None
        if cid is not None:
            phys.add((pid, cid))
    except OSError:
        pass
    return threads, (len(phys) if phys else None)


def cpu_run(case_name, budget_s, max_steps):
    """The oracle (CPU restatement of the reference step) on this host's cores: time whole steps
    of the bounded sample after its initial projection until `budget_s` or `max_steps`."""
    from oracle.oracle import Oracle
    threads, phys = host_cores()
    case, what = cpu_sample_case(case_name)
    o = Oracle(case, nthreads=threads)
    o.initialise()
    t0 = time.perf_counter()
    steps = 0
    while steps < max(1, max_steps):
        o.advance()
        steps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return dict(value=o.nc * steps / dt, unit="cell-steps/s", cores=threads, physical_cores=phys, kind="port",
                steps=steps,
                sample=f"{steps} RK3W step(s) of {what} after the initial projection, {dt:.1f} s, oracle (CPU "
                       f"restatement of the reference step, plain FP64 Jacobi-PCG) with {threads} OpenMP threads "
                       f"on {phys if phys else 'an unknown number of'} physical cores")


PROFILE = {("pcg", "channel"): "k_pcg_channel96x64x64.md", ("fcg", "channel"): "k_fcg_channel96x64x64.md",
           ("ml", "channel"): "k_mlcg_channel96x64x64.md", ("ml", "urban"): "k_mlk_urban2m.md", ("ml", "urban2m"): "k_mlk_urban2m.md"}


def pcg_traffic_per_launch(psolver, config, nc, its_per_solve):
    """DRAM bytes (read + write) of one launch of the Poisson kernel on this workload, from the
    committed ncu summary: either a capture of this workload (traffic_bytes_per_launch) or of a
    smaller mesh of the same generator, scaled by cells x iterations
    (traffic_bytes_per_cell_iteration); None when no summary exists."""
    name = PROFILE.get((psolver, config))
    if not name:
        return None
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
            if line.startswith("traffic_bytes_per_cell_iteration:"):
                return int(float(line.split(":")[1]) * nc * its_per_solve)
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
    from dopamine_b200 import abi
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
    if args.ml_value_bits:
        case.params["p_ml_value_bits"] = args.ml_value_bits
    if args.ml_degree:
        case.params["p_ml_degree"] = args.ml_degree
    if args.fcg_degree:
        case.params["p_smooth_degree"] = args.fcg_degree
    if args.host_setup:
        case.params["host_setup"] = 1
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
    # algorithmic bytes per Krylov iteration of the timed form, as the library counts them from
    # its operator and (multilevel) hierarchy
    bytes_it = s.stats()["p_bytes_per_iteration"]
    # ---- end to end through the C ABI with host buffers: the transported state (U, p, T when it
    # is transported, the passive scalars) goes up from pinned host memory and comes back every step
    L = lib()
    host = s.sync_host()
    with_T = bool(s.params.boussinesq)
    ns = max(0, min(int(s.params.n_scalars), 4))

    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

    U, p = pinned(host["U"].shape), pinned(host["p"].shape)
    U[...] = host["U"]
    p[...] = host["p"]
    T = pinned(host["T"].shape) if with_T else None
    if with_T:
        T[...] = host["T"]
    Cs = pinned((nc, ns)) if ns else None
    if ns:
        Cs[...] = s.scalars()[1].T
    dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
    bytes_per_dir = 8 * nc * (3 + 1 + (1 if with_T else 0) + ns)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = L.dpm_upload_state(s.h, dp(U), dp(p), dp(T))
        if ns:
            rc |= L.dpm_upload_scalars(s.h, dp(Cs))
        rc |= L.dpm_advance(s.h, s.params.dt)
        rc |= L.dpm_download_state(s.h, dp(U), dp(p), dp(T), None)
        if ns:
            rc |= L.dpm_download_scalars(s.h, dp(Cs))
        if rc:
            raise RuntimeError(f"e2e step failed {rc}")
    t_e2e = time.perf_counter() - t0
    clocks = sampler.stop() if sampler else None
    if world > 1:
        t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], "cuda")
    plain = None
    if args.psolver != "pcg" and not args.no_plain and world == 1:
        # the plain FP64 Jacobi-PCG form on the same handle, mesh and state: one warm-up step, then
        # `plain_steps` steps timed by the library's CUDA events
        s.select_pressure_solver(abi.PSOLVER_JACOBI_PCG)
        s.advance()
        pm, pp, pit = [], [], 0
        for _ in range(args.plain_steps):
            s.advance()
            a, b = s.last_timing()
            pm.append(a)
            pp.append(b)
            pit += s.stats()["p_iters"]
        plain = dict(ms_per_step=sum(pm) / len(pm), poisson_ms_per_step=sum(pp) / len(pp),
                     pcg_iterations_per_step=pit / len(pm), steps=len(pm))
        s.select_pressure_solver(3)
    phases = None
    if args.fcg_phases and args.psolver == "fcg":
        # diagnostics after the timed region: where an iteration of the two-level kernel goes
        s.fcg_phase_times(True)
        for _ in range(2):
            s.advance()
        phases = s.fcg_phase_times(False)
    return dict(nc=nc, t_dev=t_dev, t_e2e=t_e2e, step_ms=step_ms, pois_ms=pois_ms, its=its, solves=solves,
                bytes_it=bytes_it,
                launches=launches, clocks=clocks, solver=s, learn=learn, fallbacks=s.stats()["p_fallbacks"],
                e2e_bytes=bytes_per_dir, plain=plain, setup=s.setup_times(), phases=phases)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dopamine_b200")
    ap.add_argument("--config", default="urban", choices=list(CONFIG_NAMES))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 Jacobi-PCG form")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed steps of the plain FP64 form")
    ap.add_argument("--no-learned", action="store_true", help="flexible CG without the learned term")
    ap.add_argument("--ml-degree", type=int, default=0,
                    help="multilevel form: Chebyshev steps per smoothing (0: library default, 3)")
    ap.add_argument("--ml-value-bits", type=int, default=0, choices=[0, 16, 32],
                    help="multilevel form: storage of the smoother's scaled off-diagonals (0: library default, FP32)")
    ap.add_argument("--mixed", action="store_true", default=True,
                    help="precision form (the default: the metric is learned+mixed): FP32 gradients, SGS and flux "
                         "assembly; with the two-level form also FP32-operator inner iterations inside FP64 defect "
                         "correction")
    ap.add_argument("--fp64", action="store_true", help="the FP64 explicit half instead of the precision form")
    ap.add_argument("--fcg-degree", type=int, default=0,
                    help="Chebyshev degree of the two-level form's part-local smoother (0: library default 7)")
    ap.add_argument("--host-setup", action="store_true",
                    help="build the mesh and static operators with the host builder (reported in config.setup_ms)")
    ap.add_argument("--fcg-phases", action="store_true",
                    help="after the timed region, record the two-level kernel's phase times for 2 steps")
    ap.add_argument("--psolver", default="auto", choices=["auto", "pcg", "fcg", "ml"],
                    help="auto: fcg when the mesh fits the two-level kernel, else ml; pcg: plain FP64 "
                         "Jacobi-PCG; fcg: flexible CG, two-level part-local preconditioner; "
                         "ml: flexible CG, aggregation-multigrid V-cycle")
    args = ap.parse_args()
    if args.fp64:
        args.mixed = False

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    cfg_name = CONFIG_NAMES[args.config]

    if args.impl == "reference":
        if rank != 0:
            return 0
        # each timed step is one whole RK3W step of the bounded sample; as many of the requested
        # steps as fit in about two minutes are timed, and the line says how many
        cb = cpu_run(args.config, budget_s=120.0, max_steps=args.steps)
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": cb["steps"], "warmup": 0, "steps_requested": args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg_name, "form": "plain FP64 Jacobi-PCG (CPU restatement of the reference step)"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "physical_cores", "kind", "sample")},
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
    bytes_it = r["bytes_it"]
    pois_s = sum(r["pois_ms"]) / 1e3
    achieved = bytes_it * r["its"] / pois_s / 1e9 if pois_s > 0 else 0.0
    its_per_solve = r["its"] / max(r["solves"], 1)
    traffic = pcg_traffic_per_launch(args.psolver, args.config, nc, its_per_solve)
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": 1e3 * r["t_dev"] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32" if args.mixed else "f64", "data": "synthetic",
        "config": {"workload": cfg_name, "cells": nc, "form": FORMS[args.psolver],
                   "poisson_ms_per_step": 1e3 * pois_s / K, "pcg_iterations_per_step": r["its"] / K,
                   "poisson_solves_per_step": r["solves"] / K,
                   "l2": L2_NOTE.get(args.config, "inputs larger than L2"),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": r["e2e_bytes"],
                "d2h_bytes_per_step": r["e2e_bytes"]},
        "roofline": {"kernel": KERNELS[args.psolver], "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "bytes_per_iteration": bytes_it, "iterations_per_launch": its_per_solve},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    if args.mixed:
        line["config"]["form"] += ("; precision form: first gradient pass, SGS and flux assembly in FP32 (FP64 state, "
                                   "projection and wall-model Newton)" +
                                   ("; FP32-operator inner Krylov iterations in FP64 defect correction"
                                    if args.psolver == "fcg" else ""))
    if r["learn"] is not None:
        line["config"]["learned_term"] = r["learn"]
        g = r["learn"]["gamma"]
        line["config"]["form"] += ("; learned one-ring term (gamma %g)" % g if g > 0 else
                                   "; learned one-ring term trained, gated off (gamma 0) on the held-out solve")
    if args.psolver in ("fcg", "ml"):
        line["config"]["fallbacks_to_plain_pcg"] = r["fallbacks"]
    # handle creation (device mesh and static-operator set-up, upload, pressure-solver set-up); not timed
    line["config"]["setup_ms"] = {k: round(v, 1) for k, v in r["setup"].items()}
    if r["phases"] is not None:
        line["config"]["fcg_phase_us_per_iteration"] = {k: (round(v, 3) if isinstance(v, float) else v)
                                                        for k, v in r["phases"].items()}
    if r["plain"] is not None:
        pl = r["plain"]
        pl["speedup_of_this_form"] = pl["ms_per_step"] / line["ms_per_step"]
        line["config"]["plain_fp64_pcg"] = pl
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline is reported at N = 1 only
        cb = cpu_run(args.config, budget_s=20.0, max_steps=3)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "physical_cores", "kind", "sample")}
    print(json.dumps(line))
    s.close()
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
