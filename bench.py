#!/usr/bin/env python
"""Benchmark of the RK3 DG residual (HP-1) on one B200: the 96^3 x 6 Kuhn-tet
plane-wave workload (5,308,416 P2 tetrahedra, 6 fields, interior jitter
+/-0.15 h, random unit direction, |k| = 4 pi), FP32 residual path (FP64 setup
and norms) next to the plain FP64 path.

A step is one RK3 time step (3 fused stage kernels) over the whole mesh;
DoF-updates per step = 10 nodes x 6 fields x 3 stages x n_elements.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  With --impl reference it times the
reference's own CPU code (compiled from its sources into oracle/_ref) on this
host's cores instead.
"""
from __future__ import annotations

import argparse
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
    """Per element per RK3 step: state 60 values x (3 + 4 + 3) accesses
    (stage 0: read w, write w, write k2; stage 1: read w, k2, write w, k2;
    stage 2: read w, k2, write w), geometry 10 values and 8 ints of
    neighbour/permutation data per stage."""
    return ne * (600 * b_s + 3 * (10 * b_g + 32))


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
    r = rm.run(ref.SCHEME_RK3, ref.make_data(khat=k, kmag=kmag, pol=p), dt, steps)
    dofs = 10 * len(e) * 6 * 3 * steps
    return {"value": dofs / r["cpu_run"], "unit": "DoF-updates/s", "cores": threads,
            "kind": "reference",
            "sample": "reference dg_solve_rk3 (oracle/_ref, -O3 -fopenmp) on a %d^3x6 = %d-tet "
                      "Kuhn mesh of the same kind, %d steps, time loop only (cpu_running_t)"
                      % (n, len(e), steps)}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # warm-up sample (discarded), then the timed sample
    cpu_reference_sample(steps=max(1, min(args.warmup, 3)))
    cb = cpu_reference_sample()
    line = {"metric": "DoF-updates/s", "value": cb["value"], "unit": "DoF-updates/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "sample_n": CPU_SAMPLE_N},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "DoF-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_CUBE, help="cube resolution (default 96)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--tile", type=int, default=0, choices=[0, 32, 128],
                    help="RK3 stage kernel: 32 = warp per field, 128 = thread per element, 0 = auto")
    ap.add_argument("--only", default="both", choices=["both", "fp64", "fp32"],
                    help="profiling aid: run one precision variant only")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    pkg = load_package()
    capi, kuhn = pkg.capi, pkg.kuhn

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    W = max(3, args.warmup)
    K = args.steps
    n = args.n
    coords, e2n = kuhn.kuhn_cube(n, JITTER, seed=SEED)
    mesh = capi.mesh_build(coords, e2n)
    ne = mesh.nbelems
    dt = CFL * mesh.hmin()
    khat, kmag, pol = kuhn.random_plane_wave(SEED, KMAG)
    data = capi.plane_data(khat=khat, kmag=kmag, pol=pol)
    dofs_per_step = 10 * ne * 6 * 3
    peak, peak_kind = measured_peaks()

    results = {}
    states = {}
    for name, prec, b_s in (("fp64", capi.FP64, 8), ("fp32", capi.FP32, 4)):
        if args.only not in ("both", name):
            continue
        s = capi.Solver(mesh, capi.SCHEME_RK3, data, dt, precision=prec, device=local,
                        elems_per_cta=args.tile)
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
        err = s.error_l2()
        states[name] = s.get_state()
        results[name] = {
            "value": world * dofs_per_step / (ms * 1e-3), "ms_per_step": ms, "gpu_launches": launches,
            "l2_error_vs_analytic": err, "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg / 3,
                         "traffic": dram_traffic("rk3_stage_%s_n%d" % (name, n))},
            "solver": s}
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
        e2e = {"value": world * dofs_per_step * K / e2e_s, "unit": "DoF-updates/s",
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
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
