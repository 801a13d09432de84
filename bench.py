#!/usr/bin/env python
"""Benchmark of the D2Q9 cylinder-channel step on B200.

Workload: the cylinder channel at nx=16384, ny=4096 (67.1 M nodes; obstacle at (nx/5+1, ny/2+1),
radius ny/10+1, bounce-back walls, Poiseuille inlet, constant-density outlet, Re=100,
uMax=0.02), synthetic initial state (equilibrium at rho=1 with the Poiseuille profile).  One
step = one time step of the whole lattice.  The lattice (9.7 GB in FP64) is far larger than the
126 MB L2, so no flush is needed between steps.

Our arm (default):
  value       MLUPS of the headline kernel (--precision/--scheme, default FP64 pull), device
              time with CUDA events on the lattice's stream, max over ranks;
  e2e         the same metric through the drop-in C ABI (include/lb.h): the reference-style
              host driver (include/lbdriver.h, collide_with_stream + finalize_stream) with
              host node arrays; the timed loop includes the upload of both host arrays, the
              per-step copy-back of the two columns the driver's outlet update reads, and the
              final copy of the whole lattice back to the host;
  roofline    the dominant kernel's algorithmic bytes per launch / its measured launch time,
              against the measured HBM copy bandwidth (MEASURED_PEAKS.json);
  cpu_baseline  the reference's own OpenMP code (oracle/_ref, best variant) on a bounded
              sample of the same workload on this host's cores.
Reference arm (--impl reference): the reference's own fastest OpenMP variant, timed on this
host's cores through its own entry points on the same workload.

Multi-GPU: the step does not need a collective (independent replicas, weak scaling): each
rank advances its own lattice and the job's MLUPS is the sum over ranks of the nodes stepped
divided by the slowest rank's time.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "memory-aware-lbm_b200")
sys.path.insert(0, PKG)

# 16-bit suffixes (lbgpu.storage_form): "s" offsets from the inflow profile per row, "r"
# stochastic rounding; neither changes the bytes moved
BYTES_PER_UPDATE = {"f64": 144, "f32": 72, **{p + sfx: 36 for p in ("f16", "bf16")
                                              for sfx in ("", "s", "b", "r", "sr", "br")}}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=16384)
    p.add_argument("--ny", type=int, default=4096)
    p.add_argument("--precision", default="f64", choices=list(BYTES_PER_UPDATE))
    p.add_argument("--scheme", default="pull", choices=["pull", "aa", "pull2"],
                   help="pull2: the pull scheme with two steps per sweep (temporal blocking)")
    p.add_argument("--variants", default="auto",
                   help="comma list of precision:scheme also timed, 'auto' or 'none'")
    p.add_argument("--study", choices=["batching", "shapes", "serving", "precision"], default=None,
                   help="run a workload study instead of the headline benchmark (one GPU)")
    p.add_argument("--study-args", default="",
                   help="comma-separated key=value overrides of the study's defaults")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=20.0,
                   help="CPU budget of the cpu_baseline sample / reference arm")
    return p.parse_args()


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist, self.torch = dist, torch
            self.backend = backend

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        t = self.torch.tensor([float(v)], dtype=self.torch.float64,
                              device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        # nvidia-smi numbers GPUs physically; map through CUDA_VISIBLE_DEVICES when it is set
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.device = ids[device] if device < len(ids) else str(device)
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.25)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------------------
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key, nodes):
    """DRAM bytes per launch of a kernel from the committed ncu summary, scaled by nodes."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    k = d.get(kernel_key)
    if not k:
        return None
    return k["bytes_per_node"] * nodes


def cores_available():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cylinder(nx, ny):
    return nx // 5 + 1, ny // 2 + 1, ny // 10 + 1


def workload(nx, ny):
    """The workload label both arms print."""
    return (f"cylinder channel {nx}x{ny} ({nx * ny / 1e6:.1f}M nodes), Re=100, uMax=0.02, "
            f"bounce-back walls, constant-density outlet")


# ---------------------------------------------------------------------------------------
# the reference's own CPU code (oracle/_ref) on this host
# ---------------------------------------------------------------------------------------
def reference_cpu(nx, ny, steps_wanted, warmup, budget_s, variant=None):
    """Time the reference's OpenMP entry points; returns a dict or raises if unavailable."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.ref_available(openmp=True):
        raise RuntimeError("oracle/_ref/libref_lb_omp.so is not built")
    threads = cores_available()
    tblock = -(-nx // threads)
    c = O.Cylinder.baseline(nx, ny)
    lib = O.ref_lib(openmp=True)
    t0 = time.perf_counter()
    O.ref_setup(c, openmp=True, blk=64, tblock=tblock, nthreads=threads)
    setup_s = time.perf_counter() - t0
    candidates = [variant] if variant else ["tight", "combine", "origin", "tight_block"]
    best, best_rate = None, 0.0
    per_step = {}
    for v in candidates:   # a 2-step probe of each variant; the fastest is timed
        t0 = time.perf_counter()
        n = O.ref_step(v, 2, openmp=True)
        dt = time.perf_counter() - t0
        per_step[v] = dt / n
        if n / dt > best_rate:
            best, best_rate = v, n / dt
    w = warmup + (warmup % 2)
    if w:
        O.ref_step(best, w, openmp=True)
    est = per_step[best]
    k = max(2, min(steps_wanted, int(budget_s / est)))
    k += k % 2
    t0 = time.perf_counter()
    done = O.ref_step(best, k, openmp=True)
    dt = time.perf_counter() - t0
    lib.ref_free()
    return {"variant": best + "_openmp", "steps": done, "seconds": dt, "threads": threads,
            "mlups": nx * ny * done / dt / 1e6, "setup_s": setup_s,
            "probe_ms_per_step": {v: round(1e3 * s, 2) for v, s in per_step.items()}}


def run_reference_arm(args, dist):
    if dist.rank != 0:
        return
    nx, ny = args.nx, args.ny
    try:
        r = reference_cpu(nx, ny, args.steps, args.warmup, budget_s=150.0)
    except Exception as e:  # the reference build is missing
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    sample = (f"{r['steps']} of {args.steps} requested steps of the {nx}x{ny} channel, "
              f"reference {r['variant']} on {r['threads']} host threads")
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(r["mlups"], 2), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": r["steps"], "warmup": args.warmup,
        "ms_per_step": round(1e3 * r["seconds"] / r["steps"], 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(nx, ny), "kernel": f"reference {r['variant']} (FP64)",
                   "nodes": nx * ny, "variant": r["variant"], "parallelism": "openmp",
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": round(r["mlups"], 2), "unit": "MLUPS", "cores": r["threads"],
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(r["mlups"], 2), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "probe_ms_per_step": r["probe_ms_per_step"],
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------
def time_lattice(lbgpu, nx, ny, precision, scheme, steps, warmup, dist, sampler_dev=None):
    ox, oy, r = cylinder(nx, ny)
    base = lbgpu.storage_form(precision)[0]
    lat = lbgpu.Lattice(nx, ny, base, "pull" if scheme == "pull2" else scheme)
    try:
        if scheme == "pull2":
            lat.set_sweep_steps(2)
        lbgpu.configure_storage(lat, precision, 0.02)   # encodes the initial state: set it first
        lat.setup_cylinder(ox, oy, r, 0.02, 100.0, lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
        lat.step(warmup)
        lat.synchronize()
        dist.barrier()
        clocks = None
        if sampler_dev is not None:
            with ClockSampler(sampler_dev) as cs:
                ms = lat.step_timed(steps)
            clocks = cs.summary()
        else:
            ms = lat.step_timed(steps)
        launches = lat.last_launches
        dist.barrier()
        ms = dist.max(ms)
        return ms, launches, clocks
    finally:
        lat.close()


def step_kernel(precision, scheme):
    """The kernel that does a step of this storage and scheme (its name in the ncu launch list)."""
    half = lbgpu_storage_base(precision) in ("f16", "bf16")
    if scheme == "pull2":
        return "k_sweep2"
    if scheme == "aa":
        return "k_aa4_even/k_aa4_odd" if half else "k_aa_even/k_aa_odd"
    return "k_pull4h" if half else "k_pull"


def lbgpu_storage_base(precision):
    """'f16sr' -> 'f16' without importing the library (used for labels only)."""
    for base in ("bf16", "f16", "f32", "f64"):
        if precision.startswith(base):
            return base
    return precision


def run_ours(args, dist):
    import lbgpu

    nx, ny, K, W = args.nx, args.ny, args.steps, max(3, args.warmup)
    dev = dist.local
    rc = lbgpu.lib().lbgpu_set_device(dev)
    if rc != 0:
        raise lbgpu.LbError(rc, lbgpu.last_error()[1])
    nodes = nx * ny
    ms, launches, clocks = time_lattice(lbgpu, nx, ny, args.precision, args.scheme, K, W, dist,
                                        sampler_dev=dev)
    per_launch_s = ms * 1e-3 / K
    mlups = dist.world * nodes * K / (ms * 1e-3) / 1e6
    peak, peak_kind = measured_peaks()
    bpu = BYTES_PER_UPDATE[args.precision]
    achieved = bpu * nodes / per_launch_s / 1e9
    key = f"{args.precision}_{args.scheme}"
    traffic = ncu_traffic(key, nodes)

    variants = {}
    vlist = []
    if args.variants == "auto":
        vlist = [("f64", "aa"), ("f64", "pull2"), ("f32", "pull"), ("f32", "aa"), ("f32", "pull2"),
                 ("f16", "pull"), ("bf16", "pull"), ("f16", "aa"), ("f16", "pull2"),
                 ("f16r", "pull"), ("f16sr", "pull"), ("f16br", "pull"), ("f16r", "aa")]
    elif args.variants != "none":
        vlist = [tuple(v.split(":")) for v in args.variants.split(",") if v]
    for prec, sch in vlist:
        if (prec, sch) == (args.precision, args.scheme):
            continue
        try:
            vms, vl, _ = time_lattice(lbgpu, nx, ny, prec, sch, K, W, dist)
            vb = BYTES_PER_UPDATE[prec]
            variants[f"{prec}_{sch}"] = {
                "mlups": round(dist.world * nodes * K / (vms * 1e-3) / 1e6, 1),
                "ms_per_step": round(vms / K, 4),
                "gbs_algorithmic": round(vb * nodes / (vms * 1e-3 / K) / 1e9, 1),
                "roofline_frac": round(vb * nodes / (vms * 1e-3 / K) / 1e9 / peak, 4)}
            if sch == "pull2":   # its own algorithmic bytes: one read + one write per two steps
                variants[f"{prec}_{sch}"]["own_bytes_per_update"] = vb // 2
                variants[f"{prec}_{sch}"]["own_roofline_frac"] = round(
                    vb / 2 * nodes / (vms * 1e-3 / K) / 1e9 / peak, 4)
        except Exception as e:  # a kernel family not built yet is reported, not hidden
            variants[f"{prec}_{sch}"] = {"error": str(e)[:200]}

    e2e = None
    if not args.no_e2e:
        ox, oy, r = cylinder(nx, ny)
        dist.barrier()
        _, done, secs = lbgpu.drive(nx, ny, ox, oy, r, K, "combine", wall=lbgpu.WALL_BOUNCEBACK,
                                    outlet=lbgpu.OUTLET_CONST, sync="outlet", want_lattice=False)
        secs = dist.max(secs)
        # bytes the library copied (lbdrv_last_transfer_bytes): the first call's upload of the
        # current lattice, the second buffer's ghost ring and perimeter bands, the dynamics tags
        # and tables; the outlet columns after every step; the final copy-back
        h2d, d2h = lbgpu.drive_transfer_bytes()
        e2e = {"value": round(dist.world * nodes * done / secs / 1e6, 1), "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d / done), "d2h_bytes_per_step": int(d2h / done),
               "seconds": round(secs, 3), "steps": done,
               "path": "lb.h drop-in: collide_with_stream + finalize_stream, host node arrays"}

    cpu = None
    if not args.no_cpu_baseline and dist.rank == 0 and dist.world == 1:
        try:
            r = reference_cpu(nx, ny, 10**9, 0, budget_s=args.cpu_seconds)
            cpu = {"value": round(r["mlups"], 2), "unit": "MLUPS", "cores": r["threads"],
                   "kind": "reference",
                   "sample": f"{r['steps']} steps of the {nx}x{ny} channel, reference "
                             f"{r['variant']} (fastest of a 2-step probe)"}
        except Exception as e:
            cpu = {"value": None, "unit": "MLUPS", "cores": cores_available(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    line = {
        "metric": "MLUPS", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": dist.world,
        "steps": K, "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": workload(nx, ny),
                   "kernel": f"{step_kernel(args.precision, args.scheme)} "
                             f"({args.precision.upper()} {args.scheme})",
                   "nodes_per_gpu": nodes, "l2": "inputs larger than L2 (lattice "
                   f"{bpu * nodes / 1e9:.1f} GB streamed per step)",
                   "parallelism": f"replicas x{dist.world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": None if traffic is None else int(traffic),
                     "kernel": f"{step_kernel(args.precision, args.scheme)} ({args.precision})",
                     "bytes_per_update": bpu, "peak_kind": f"{peak_kind} hbm_gbs (copy)"},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "variants": variants,
    }
    if dist.rank == 0:
        print(json.dumps(line))


def run_study(args, dist):
    """One study on this rank's GPU (rank 0 prints; the studies are single-GPU workloads)."""
    import lbgpu
    import studies

    rc = lbgpu.lib().lbgpu_set_device(dist.local)
    if rc != 0:
        raise lbgpu.LbError(rc, lbgpu.last_error()[1])
    kw = {}
    for item in filter(None, args.study_args.split(",")):
        k, v = item.split("=", 1)
        if "/" in v or k in ("precisions", "cases"):
            kw[k] = tuple(v.split("/"))
        else:
            try:
                kw[k] = int(v)
            except ValueError:
                kw[k] = float(v) if v.replace(".", "", 1).replace("e-", "", 1).isdigit() else v
    if dist.rank != 0:
        return
    fn = {"batching": studies.batching_study, "shapes": studies.member_shape_study,
          "serving": studies.serving_study, "precision": studies.precision_study}[args.study]
    t0 = time.time()
    with ClockSampler(dist.local) as cs:
        res = fn(**kw)
    res = {"study": args.study, "args": {k: list(v) if isinstance(v, tuple) else v
                                         for k, v in kw.items()},
           "wall_s": round(time.time() - t0, 1), "clocks": cs.summary(), **res}
    print(json.dumps(res))


def main():
    args = parse()
    dist = Dist()
    try:
        if args.study:
            run_study(args, dist)
        elif args.impl == "reference":
            run_reference_arm(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
