#!/usr/bin/env python
"""Benchmarks of the two hot paths on one B200.  Prints one JSON line (rank 0).

--workload rk3 (default, the headline): the RK3 DG residual (HP-1) on the
  96^3 x 6 Kuhn-tet plane-wave workload (5,308,416 P2 tetrahedra, 6 fields,
  interior jitter +/-0.15 h, random unit direction, |k| = 4 pi), FP32 residual
  path (FP64 setup and norms) next to the plain FP64 path.  A step is one RK3
  time step (3 fused stage kernels) over the whole mesh; DoF-updates per step
  = 10 nodes x 6 fields x 3 stages x n_elements.
--workload kinetic: the CFL-less precision study (HP-2) on the 64^3 x 6 PEC
  cavity, d3q4, dt = 20 x the RK3 CFL step: FP64, FP32 sweeps, FP32 sweeps +
  1 and 2 FP64-residual refinements, BF16 distributions.  DoF-updates per step
  = 10 nodes x 24 kinetic components x n_elements.
--workload batched: 256 independent plane-wave solves of uneven size (n in
  [8, 40], jitter 0.1 h, random direction, |k| in [2 pi, 8 pi]): 128 RK3 (100
  steps) and 128 CFL-less at 10 x CFL (10 steps), FP32, each scheme's
  instances in one batch handle, both batches on concurrent streams; against
  the instances run one at a time on the plain FP64 path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload rk3|kinetic|batched]

With --impl reference it times the reference's own CPU code (compiled from
its sources into oracle/_ref) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import contextlib
import ctypes
import multiprocessing
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dg-cfl-less-maxwell-solver_b200")

N_CUBE = 96
JITTER = 0.15
SEED = 2026
KMAG = 4.0 * np.pi
CFL = 0.3
# CPU sample of the same workload for the reference: a 12^3 x 6 mesh
CPU_SAMPLE_N = 12
CPU_SAMPLE_STEPS = 20
WORKLOAD = "rk3-planewave-kuhn96x6-jitter0.15"
# kinetic precision study: 64^3 x 6 cavity, d3q4, 20 x CFL
KIN_N = 64
KIN_MULT = 20
KIN_STEPS = 100
KIN_WORKLOAD = "kinetic-cavity-d3q4-kuhn64x6-20xcfl"
KIN_CPU_N = 8
# batched uneven workload
BATCH_COUNT = 256
BATCH_RK3_STEPS = 100
BATCH_KIN_STEPS = 10
BATCH_KIN_MULT = 10
BATCH_WORKLOAD = "batched-256-planewave-kuhn8to40-rk3x100-kineticx10"


def load_package():
    if "gdon3d_b200" in sys.modules:
        return sys.modules["gdon3d_b200"]
    spec = importlib.util.spec_from_file_location(
        "gdon3d_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gdon3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic(kernel_key):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(kernel_key)
    return None if v is None else float(v["bytes_per_launch"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([t.strip() for t in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        pw = [float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None,
                "samples": len(self.rows), "reasons": sorted(reasons)}


def algorithmic_bytes_per_step(ne, b_s, b_g):
    """The per-element figure of the hot-path scope, per RK3 step: state 60
    values x (3 + 4 + 4) accesses (stage 0: read w, write w, write k2; stages
    1 and 2: read w, k2, write w, k2), geometry 10 values and 20 bytes of
    connectivity per stage: 660 b_s + 30 b_g + 60."""
    return ne * (660 * b_s + 30 * b_g + 60)


def tight_bytes_per_step(ne, b_s, b_g):
    """What this kernel must move at least: k2 is dead after the last stage and
    is not written there (600 b_s), and each stage reads 32 bytes of neighbour
    and permutation records."""
    return ne * (600 * b_s + 3 * (10 * b_g + 32))


@contextlib.contextmanager
def c_stdout_to_stderr():
    """The reference's time loops print progress to the C stdout ("\\r[Info]
    t = ..."); send file descriptor 1 to stderr meanwhile, so that stdout
    carries only the JSON line."""
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def cpu_reference_sample(steps=CPU_SAMPLE_STEPS, n=CPU_SAMPLE_N):
    """The reference's own RK3 (oracle/_ref) on this host's cores, all threads."""
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, ROOT)
    from oracle import ref
    gk = load_package().kuhn
    c, e = gk.kuhn_cube(n, JITTER, seed=SEED)
    k, kmag, p = gk.random_plane_wave(SEED, KMAG)
    rm = ref.RefMesh(c, e)
    dt = CFL * rm.hmin()
    with c_stdout_to_stderr():
        r = rm.run(ref.SCHEME_RK3, ref.make_data(khat=k, kmag=kmag, pol=p), dt, steps)
    dofs = 10 * len(e) * 6 * 3 * steps
    return {"value": dofs / r["cpu_run"], "unit": "DoF-updates/s", "cores": threads,
            "kind": "reference",
            "sample": "reference dg_solve_rk3 (oracle/_ref, -O3 -fopenmp) on a %d^3x6 = %d-tet "
                      "Kuhn mesh of the same kind, %d steps, time loop only (cpu_running_t)"
                      % (n, len(e), steps)}


def cpu_reference_kinetic_sample(steps=10, n=KIN_CPU_N):
    """The reference's own CFL-less solve (oracle/_ref: SpMV + sparse LU per
    velocity and field, then the relaxation) on this host's cores."""
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, ROOT)
    from oracle import ref
    gk = load_package().kuhn
    c, e = gk.kuhn_cube(n, 0.0, seed=SEED)
    rm = ref.RefMesh(c, e)
    dt = KIN_MULT * CFL * rm.hmin()
    with c_stdout_to_stderr():
        r = rm.run(ref.SCHEME_D3Q4, ref.make_data(kind=ref.DATA_CAVITY), dt, steps)
    dofs = 10 * len(e) * 24 * steps
    return {"value": dofs / r["cpu_run"], "unit": "DoF-updates/s", "cores": threads, "kind": "reference",
            "sample": "reference dg_solve_relaxation (oracle/_ref, -O3 -fopenmp) on a %d^3x6 = %d-tet cavity "
                      "mesh, d3q4, %dx CFL, %d steps, time loop only; its sparse solves run the oracle's "
                      "block-triangular direct LU (oracle/shim/sparse_shim.c), not SuiteSparse KLU, which "
                      "is not installed"
                      % (n, len(e), KIN_MULT, steps)}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "kinetic":
        cpu_reference_kinetic_sample(steps=1)
        cb = cpu_reference_kinetic_sample()
        wl = KIN_WORKLOAD
    else:
        # warm-up sample (discarded), then the timed sample; the batched
        # workload's reference arm is the same RK3 sample (the instances'
        # dominant scheme)
        cpu_reference_sample(steps=max(1, min(args.warmup, 3)))
        cb = cpu_reference_sample()
        wl = WORKLOAD if args.workload == "rk3" else BATCH_WORKLOAD
    line = {"metric": "DoF-updates/s", "value": cb["value"], "unit": "DoF-updates/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": wl, "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "DoF-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _build_instance_mesh(spec):
    """Worker (spawned process, no GPU): the T4 mesh and its connectivity."""
    pkg = load_package()
    c, e = pkg.kuhn.kuhn_cube(spec["n"], spec["jitter"], seed=spec["jitter_seed"])
    m = pkg.capi.mesh_build(c, e)
    return (m.face2elem, m.fnode2enode, m.boundaryface, m.elem2qnode, m.node, m.nbelems, m.hmin())


def max_over_ranks(dist, x: float, device) -> float:
    """The slowest rank's time: every rank times its own replica on the
    device; the job takes as long as the slowest one."""
    import torch
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput of `world` replicas (weak scaling): the units all
    ranks processed over the slowest rank's time."""
    return world * units_per_rank / seconds


class Env:
    """Process-group plumbing shared by the workloads (one process per GPU,
    NCCL; the workloads run one replica per rank, no data-path collective)."""

    def __init__(self, args):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        if self.world > 1:
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", device_id=torch.device("cuda", self.local),
                                    timeout=__import__("datetime").timedelta(seconds=600))
        torch.cuda.set_device(self.local)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max_over_ranks(self, x):
        return max_over_ranks(self.dist, x, "cuda")

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 50 rk3, 100 kinetic; batched runs its fixed step counts)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rk3", choices=["rk3", "kinetic", "batched"])
    ap.add_argument("--n", type=int, default=None, help="cube resolution (default 96 rk3, 64 kinetic)")
    ap.add_argument("--count", type=int, default=BATCH_COUNT, help="batched: number of instances")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--variant", type=int, default=0, choices=[0, 1, 2],
                    help="RK3 stage kernel: 1 / 2 = compiled for fewer / more resident CTAs per SM, "
                         "0 = autotuned")
    ap.add_argument("--only", default="all",
                    help="profiling aid: comma-separated variants to run (rk3: fp64,fp32; kinetic: "
                         "fp64,fp32,fp32_refine1,fp32_refine2,bf16)")
    ap.add_argument("--kin-sweep", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="kinetic: force the sweep mode (1 level launches, 2 cooperative, 3 readiness "
                         "flags, 4 spatial parts) and skip the per-mode timing; 0 = autotuned, with the "
                         "per-mode timing")
    ap.add_argument("--headline-only", action="store_true",
                    help="rk3: print the 96^3 line without the kinetic precision study and the batch")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = {"rk3": 50, "kinetic": KIN_STEPS, "batched": BATCH_RK3_STEPS}[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args)
    with_all = args.workload == "rk3" and not args.headline_only and args.n is None
    specs = built = None
    if args.workload == "batched" or with_all:
        # meshes first, in spawned worker processes (no CUDA in them)
        specs = load_package().kuhn.uneven_plane_wave_batch(SEED, args.count)
        ctx = multiprocessing.get_context("spawn")
        with concurrent.futures.ProcessPoolExecutor(max_workers=min(32, os.cpu_count() or 1),
                                                    mp_context=ctx) as ex:
            built = list(ex.map(_build_instance_mesh, specs, chunksize=4))
    env = Env(args)
    if args.workload == "batched":
        line = run_batched(args, env, specs, built)
    elif args.workload == "kinetic":
        line = run_kinetic(args, env)
    else:
        line = run_rk3(args, env)
        if with_all:
            # configs 4 and 5 ride on the default line, each with its own
            # clocks and roofline: the 64^3 kinetic precision study (100
            # steps per variant) and the 256-instance uneven batch
            kargs = argparse.Namespace(**vars(args))
            kargs.steps = KIN_STEPS
            kargs.n = None
            kargs.only = "all"
            line["kinetic_precision_study"] = _strip(run_kinetic(kargs, env))
            line["batched_uneven_256"] = _strip(run_batched(args, env, specs, built))
    if env.rank == 0:
        print(json.dumps(line), flush=True)
    env.close()
    return 0


def _strip(line):
    """A sub-benchmark's line as a key of the default line: its own metric,
    value, config, roofline, clocks and variants, without the keys that only
    the top-level line carries."""
    return {k: v for k, v in line.items()
            if k not in ("n_gpus", "vs_baseline", "e2e", "e2e_note", "data", "scaling", "higher_is_better")}


def _wanted(args, name):
    return args.only == "all" or name in args.only.split(",")


def run_rk3(args, env):
    torch = env.torch
    world, rank, local = env.world, env.rank, env.local
    barrier, max_over_ranks = env.barrier, env.max_over_ranks
    pkg = load_package()
    capi, kuhn = pkg.capi, pkg.kuhn

    W = max(3, args.warmup)
    K = args.steps
    n = args.n or N_CUBE
    coords, e2n = kuhn.kuhn_cube(n, JITTER, seed=SEED)
    mesh = capi.mesh_build(coords, e2n, device=local)
    ne = mesh.nbelems
    dt = CFL * mesh.hmin()
    khat, kmag, pol = kuhn.random_plane_wave(SEED, KMAG)
    data = capi.plane_data(khat=khat, kmag=kmag, pol=pol)
    dofs_per_step = 10 * ne * 6 * 3
    peak, peak_kind = measured_peaks()

    results = {}
    states = {}
    for name, prec, b_s in (("fp64", capi.FP64, 8), ("fp32", capi.FP32, 4)):
        if not _wanted(args, name):
            continue
        s = capi.Solver(mesh, capi.SCHEME_RK3, data, dt, precision=prec, device=local,
                        rk3_variant=args.variant)
        st = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", local))
        s.init()
        s.advance(W)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        l0 = s.launches
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ev0.record(st)
            s.advance(K)
            ev1.record(st)
            torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(ev0.elapsed_time(ev1)) / K
        launches = s.launches - l0
        alg = algorithmic_bytes_per_step(ne, b_s, b_s)
        achieved = alg / 3 / (ms / 3 * 1e-3) / 1e9  # per launch bytes / launch time
        tight = tight_bytes_per_step(ne, b_s, b_s) / (ms * 1e-3) / 1e9
        err = s.error_l2()
        states[name] = s.get_state()
        results[name] = {
            "value": job_rate(world, dofs_per_step, ms * 1e-3), "ms_per_step": ms, "gpu_launches": launches,
            "l2_error_vs_analytic": err, "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg / 3,
                         "achieved_tight_count": tight, "frac_tight_count": tight / peak,
                         "traffic": dram_traffic("rk3_stage_%s_n%d" % (name, n))},
            "rk3_variant": s.rk3_variant, "solver": s}
    rel_fp32 = None
    if "fp64" in states and "fp32" in states:
        ref64 = states["fp64"][: 60 * ne]
        rel_fp32 = float(np.linalg.norm(states["fp32"][: 60 * ne] - ref64) / np.linalg.norm(ref64))
    head = results["fp32"] if "fp32" in results else results["fp64"]

    # e2e through the C-ABI with host buffers: one gdn_cuda_step_host call of K
    # steps (H2D of the reference-layout state from pinned memory, K steps, D2H)
    e2e = None
    if not args.no_e2e:
        sh = head["solver"]
        wl = sh.wlen
        host = torch.empty(wl, dtype=torch.float64, pin_memory=True)
        hv = host.numpy()
        hv[:] = states["fp32" if "fp32" in states else "fp64"]
        sh.step_host(hv, 1)  # warm the host path
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sh.step_host(hv, K)
        t1 = time.perf_counter()
        barrier()
        e2e_s = max_over_ranks(t1 - t0)
        e2e = {"value": job_rate(world, dofs_per_step * K, e2e_s), "unit": "DoF-updates/s",
               "h2d_bytes_per_step": wl * 8 / K, "d2h_bytes_per_step": wl * 8 / K,
               "call": "gdn_cuda_step_host: reference-layout FP64 state in pinned host memory, "
                       "copied in, %d steps, copied out" % K}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_sample()
        except Exception as ex:  # the reference build is test infrastructure
            cpu = {"value": None, "unit": "DoF-updates/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "unavailable: %s" % ex}

    for r in results.values():
        r.pop("solver").close()
    line = {
        "metric": "DoF-updates/s", "value": head["value"], "unit": "DoF-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if "fp32" in results else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD if n == N_CUBE else WORKLOAD.replace("96", str(n)),
                   "n_elements": ne, "p": 2, "fields": 6, "steps_timed": K,
                   "dt": dt, "cfl": CFL, "seed": SEED, "khat": list(map(float, khat)), "kmag": kmag,
                   "precision": "FP32 state and residual arithmetic; FP64 geometry setup and norms",
                   "l2_flush": "inputs larger than L2: FP32 state %.2f GB per buffer vs 126 MB L2"
                               % (60 * ne * 4 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single-gpu"},
        "roofline": head["roofline"], "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
        "rk3_variant": head["rk3_variant"],
        "l2_rel_fp32_vs_fp64": rel_fp32,
        "l2_error_vs_analytic": {k: v["l2_error_vs_analytic"] for k, v in results.items()},
        "variants": {k + ("_plain" if k == "fp64" else ""):
                     {q: v[q] for q in ("value", "ms_per_step", "roofline", "clocks", "gpu_launches")}
                     for k, v in results.items()},
        "speedup_fp32_vs_fp64": (results["fp32"]["value"] / results["fp64"]["value"]
                                 if len(results) == 2 else None),
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    return line




def _time_advance(env, solver, steps, device):
    """Device time (ms) of `steps` steps on the solver's stream, and the
    kernels launched, with the clocks sampled meanwhile."""
    torch = env.torch
    st = torch.cuda.ExternalStream(solver.stream, device=torch.device("cuda", device))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = solver.launches
    env.barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        ev0.record(st)
        solver.advance(steps)
        ev1.record(st)
        torch.cuda.synchronize()
    env.barrier()
    return env.max_over_ranks(ev0.elapsed_time(ev1)), solver.launches - l0, clk.summary()


def kinetic_algorithmic_bytes(ne, b_s, b_g):
    """Minimum traffic of a CFL-less step per element: read f^n and write
    f^{n+1} once (240 values each), the geometry (10 values) and 20 bytes of
    connectivity; factors, levels and refinement are implementation traffic."""
    return ne * (2 * 240 * b_s + 10 * b_g + 20)


def run_kinetic(args, env):
    torch = env.torch
    pkg = load_package()
    capi, kuhn = pkg.capi, pkg.kuhn
    W = max(3, args.warmup)
    K = args.steps
    n = args.n or KIN_N
    c, e = kuhn.kuhn_cube(n, 0.0, seed=SEED)
    mesh = capi.mesh_build(c, e, device=env.local)
    ne = mesh.nbelems
    dt = KIN_MULT * CFL * mesh.hmin()
    data = capi.cavity_data()
    dofs_per_step = 10 * ne * 24
    peak, peak_kind = measured_peaks()
    variants = [("fp64", capi.FP64, 1, 8, 8), ("fp32", capi.FP32, 1, 4, 4),
                ("fp32_refine1", capi.FP32_REFINE, 1, 8, 4), ("fp32_refine2", capi.FP32_REFINE, 2, 8, 4),
                ("bf16", capi.BF16_STORE, 1, 2, 4)]
    res = {}
    ref_state = None
    vol = None
    for name, prec, passes, b_s, b_g in variants:
        if not _wanted(args, name):
            continue
        s = capi.Solver(mesh, capi.SCHEME_KINETIC, data, dt, precision=prec, refine_passes=passes, nb_v=4,
                        device=env.local, kin_sweep=args.kin_sweep)
        s.init()
        s.advance(W)  # warm-up, captures the step graph
        s.init()
        ms, launches, clk = _time_advance(env, s, K, env.local)
        ms /= K
        err = s.error_l2()
        wn = s.get_state()
        levels = s.num_levels
        mode = s.kin_sweep_mode
        s.close()
        if vol is None:
            vol = np.zeros((24, len(wn) // 24), bool)
            vol[:, : 10 * ne] = True
            vol = vol.ravel()
        if name == "fp64":
            ref_state = wn[vol]
            rel = 0.0
        elif ref_state is not None:
            rel = float(np.linalg.norm(wn[vol] - ref_state) / np.linalg.norm(ref_state))
        else:
            rel = None  # FP64 reference variant not run (--only)
        del wn
        alg = kinetic_algorithmic_bytes(ne, b_s, b_g)
        achieved = alg / (ms * 1e-3) / 1e9
        res[name] = {"value": job_rate(env.world, dofs_per_step, ms * 1e-3), "ms_per_step": ms,
                     "gpu_launches": launches, "levels": levels, "sweep_mode": mode, "clocks": clk,
                     "l2_rel_vs_fp64": rel, "l2_error_vs_analytic": err,
                     "roofline": {"bound": "hbm", "scope": "whole step vs the minimum traffic",
                                  "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                                  "peak_kind": peak_kind, "algorithmic_bytes_per_step": alg}}
    # the three sweep-level groupings of the transport solve, timed alone
    # (the variants above run the one the autotuner picked)
    sweep_modes = {}
    for name, prec in (("fp64", capi.FP64), ("fp32", capi.FP32)):
        if not _wanted(args, name) or args.kin_sweep:
            continue
        sweep_modes[name] = {}
        for mode, label in ((1, "level_launches"), (2, "cooperative_grid_barrier"), (3, "readiness_flags"),
                            (4, "spatial_parts")):
            s = capi.Solver(mesh, capi.SCHEME_KINETIC, data, dt, precision=prec, nb_v=4, device=env.local,
                            kin_sweep=mode)
            s.init()
            s.advance(W)
            s.init()
            ms, launches, _ = _time_advance(env, s, min(K, 20), env.local)
            s.close()
            sweep_modes[name][label] = {"ms_per_step": ms / min(K, 20), "gpu_launches_per_step":
                                        launches / min(K, 20)}
    if "fp64" in res:
        e64 = res["fp64"]["l2_error_vs_analytic"]
        for r in res.values():
            r["analytic_error_vs_fp64_pct"] = 100.0 * (r["l2_error_vs_analytic"] - e64) / e64
        ok = [k for k, r in res.items() if abs(r["analytic_error_vs_fp64_pct"]) <= 1.0]
    else:
        ok = list(res)
    best = max(ok, key=lambda k: res[k]["value"])
    cpu = None
    if env.rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_kinetic_sample()
        except Exception as ex:
            cpu = {"value": None, "unit": "DoF-updates/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "unavailable: %s" % ex}
    head = res[best]
    line = {
        "metric": "DoF-updates/s", "value": head["value"], "unit": "DoF-updates/s", "n_gpus": env.world,
        "steps": K, "warmup": W, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": {"fp64": "f64", "bf16": "bf16"}.get(best, "f32"),
        "data": "synthetic",
        "config": {"workload": KIN_WORKLOAD if n == KIN_N else KIN_WORKLOAD.replace("64", str(n)),
                   "n_elements": ne, "velocities": 4, "dt": dt, "cfl_multiple": KIN_MULT,
                   "headline_variant": best,
                   "headline_rule": "fastest variant whose analytic L2 error is within 1% of the FP64 one",
                   "l2_flush": "inputs larger than L2: %.2f GB of distributions" % (ne * 240 * 4 / 1e9),
                   "parallelism": "replicas" if env.world > 1 else "single-gpu"},
        "roofline": head["roofline"], "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
        "variants": res, "sweep_modes": sweep_modes, "e2e": None,
        "e2e_note": "the end-to-end line is the default (rk3) workload's",
        "cpu_baseline": cpu,
    }
    return line


def run_batched(args, env, specs, built):
    torch = env.torch
    pkg = load_package()
    capi = pkg.capi
    W = max(3, args.warmup)
    meshes = [capi.MeshArrays(*b[:6]) for b in built]
    hmins = [b[6] for b in built]
    datas = [capi.plane_data(khat=sp["khat"], kmag=sp["kmag"], pol=sp["pol"]) for sp in specs]
    rk = [i for i, sp in enumerate(specs) if sp["scheme"] == "rk3"]
    kn = [i for i, sp in enumerate(specs) if sp["scheme"] == "kinetic"]
    dts = [(CFL if specs[i]["scheme"] == "rk3" else BATCH_KIN_MULT * CFL) * hmins[i] for i in range(len(specs))]
    ne = [m.nbelems for m in meshes]
    dofs_rk = sum(10 * ne[i] * 18 * BATCH_RK3_STEPS for i in rk)
    dofs_kn = sum(10 * ne[i] * 24 * BATCH_KIN_STEPS for i in kn)
    dev = torch.device("cuda", env.local)

    # ---- batched, FP32: one handle per scheme, both on concurrent streams
    t0 = time.perf_counter()
    brk = capi.BatchSolver([meshes[i] for i in rk], [datas[i] for i in rk], [dts[i] for i in rk],
                           scheme=capi.SCHEME_RK3, precision=capi.FP32, device=env.local)
    bkn = capi.BatchSolver([meshes[i] for i in kn], [datas[i] for i in kn], [dts[i] for i in kn],
                           scheme=capi.SCHEME_KINETIC, precision=capi.FP32, nb_v=4, device=env.local)
    attach_s = time.perf_counter() - t0
    for b in (brk, bkn):
        b.init()
        b.advance(W)  # warm-up, captures the step graphs
    torch.cuda.synchronize()
    alone = {}
    for name, b, steps in (("rk3", brk, BATCH_RK3_STEPS), ("kinetic", bkn, BATCH_KIN_STEPS)):
        b.init()
        ms, launches, clk = _time_advance(env, b, steps, env.local)
        alone[name] = {"ms": ms, "gpu_launches": launches, "clocks": clk}
    brk.init()
    bkn.init()
    sa = torch.cuda.ExternalStream(brk.stream, device=dev)
    sb = torch.cuda.ExternalStream(bkn.stream, device=dev)
    ev0, eva, evb = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    l0 = brk.launches + bkn.launches
    env.barrier()
    torch.cuda.synchronize()
    with ClockSampler(env.local) as clk:
        ev0.record(sa)
        sb.wait_event(ev0)
        brk.advance(BATCH_RK3_STEPS)
        bkn.advance(BATCH_KIN_STEPS)
        eva.record(sa)
        evb.record(sb)
        torch.cuda.synchronize()
    env.barrier()
    ms_batch = env.max_over_ranks(max(ev0.elapsed_time(eva), ev0.elapsed_time(evb)))
    launches = brk.launches + bkn.launches - l0
    err_b = {"rk3": brk.error_l2_batch(), "kinetic": bkn.error_l2_batch()}
    tile = brk.rk3_variant
    levels = bkn.num_levels
    kmode = bkn.kin_sweep_mode
    brk.close()
    bkn.close()
    value = job_rate(env.world, dofs_rk + dofs_kn, ms_batch * 1e-3)

    # ---- the same instances one at a time on the plain FP64 path
    ms_single = 0.0
    err_s = {"rk3": [], "kinetic": []}
    for i, sp in enumerate(specs):
        scheme = capi.SCHEME_RK3 if sp["scheme"] == "rk3" else capi.SCHEME_KINETIC
        steps = BATCH_RK3_STEPS if sp["scheme"] == "rk3" else BATCH_KIN_STEPS
        s = capi.Solver(meshes[i], scheme, datas[i], dts[i], precision=capi.FP64, nb_v=4, device=env.local)
        s.init()
        s.advance(2)  # warm-up, captures the step graph
        s.init()
        torch.cuda.synchronize()
        st = torch.cuda.ExternalStream(s.stream, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.advance(steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms_single += e0.elapsed_time(e1)
        err_s[sp["scheme"]].append(s.error_l2())
        s.close()
    ms_single = env.max_over_ranks(ms_single)
    single_value = job_rate(env.world, dofs_rk + dofs_kn, ms_single * 1e-3)
    dev_pct = {}
    for k in ("rk3", "kinetic"):
        a, b = np.asarray(err_b[k]), np.asarray(err_s[k])
        dev_pct[k] = float(np.max(np.abs(a - b) / b) * 100.0)
    peak, peak_kind = measured_peaks()
    rk_alg = sum(algorithmic_bytes_per_step(ne[i], 4, 4) for i in rk)
    rk_achieved = rk_alg / (alone["rk3"]["ms"] / BATCH_RK3_STEPS * 1e-3) / 1e9
    line = {
        "metric": "DoF-updates/s", "value": value, "unit": "DoF-updates/s", "n_gpus": env.world,
        "steps": BATCH_RK3_STEPS, "warmup": W, "ms_per_step": ms_batch / BATCH_RK3_STEPS,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD if args.count == BATCH_COUNT else
                   BATCH_WORKLOAD.replace("256", str(args.count)),
                   "instances": len(specs), "rk3_instances": len(rk), "kinetic_instances": len(kn),
                   "elements_total": int(sum(ne)), "rk3_elements": int(sum(ne[i] for i in rk)),
                   "kinetic_elements": int(sum(ne[i] for i in kn)), "n_range": [8, 40], "jitter": 0.1,
                   "seed": SEED, "rk3_steps": BATCH_RK3_STEPS, "kinetic_steps": BATCH_KIN_STEPS,
                   "kinetic_cfl_multiple": BATCH_KIN_MULT, "rk3_variant_autotuned": tile,
                   "kinetic_sweep_mode_autotuned": {1: "level_launches", 2: "cooperative_grid_barrier",
                                                    3: "readiness_flags", 4: "spatial_parts"}.get(kmode, kmode),
                   "kinetic_levels": levels, "attach_s": attach_s,
                   "precision": "FP32 state and arithmetic; FP64 setup and norms",
                   "l2_flush": "inputs larger than L2 (%.1f GB of FP32 RK3 state)"
                               % (sum(ne[i] for i in rk) * 720 / 1e9),
                   "parallelism": "replicas" if env.world > 1 else "single-gpu"},
        "ms_total": ms_batch, "gpu_launches": launches, "clocks": clk.summary(),
        "alone_ms": {k: v["ms"] for k, v in alone.items()},
        "overlap_gain": (alone["rk3"]["ms"] + alone["kinetic"]["ms"]) / ms_batch,
        "roofline": {"bound": "hbm", "scope": "RK3 batch alone, 3 stage launches per step",
                     "achieved": rk_achieved, "peak": peak, "unit": "GB/s", "frac": rk_achieved / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_step": rk_alg},
        "one_at_a_time_fp64": {"value": single_value, "ms_total": ms_single},
        "speedup_vs_one_at_a_time_fp64": value / single_value,
        "analytic_error_fp32_batch_vs_fp64_single_max_pct": dev_pct,
        "e2e": None, "e2e_note": "the end-to-end line is the default (rk3) workload's",
        "cpu_baseline": None,
    }
    return line


if __name__ == "__main__":
    sys.exit(main())
