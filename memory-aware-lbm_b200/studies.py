"""Workload studies behind `bench.py --study`: batching, serving and storage precision.

Every number comes from the library's kernels through lbgpu.py; the inputs are seeded synthetic
cylinder channels (bounce-back walls, Poiseuille inlet, constant-density outlet).

batching   independent channels of uneven size, Reynolds number and obstacle placement stepped
           together (one launch per work list and step, persistent or one block per strip as
           the autotuner picks, CUDA-graph chunks of 50 steps, tile shapes and pull/AA chosen per
           size class by the autotuners) against a sequential loop that steps each channel
           alone with its own launches.
shapes     the batch's speed against its members' size and shape at a constant node count:
           one large channel stepped alone, then batches of equal members, from one member of
           the whole size down to many small ones, and members of equal area from wide and
           short to narrow and tall.
serving    a Poisson stream of channel requests through lbgpu_server: continuous batching under
           an HBM budget against sequential plain solves of the same requests; p50/p99 latency,
           aggregate MLUPS, and the velocity error of a sample against FP64 re-runs.
precision  one large channel stored as FP16 or BF16 offsets (from w_i, or with the suffix "s"
           from the inflow profile's equilibrium per row) against the FP64 kernel: relative L2
           error of the time-averaged velocity, mass drift, drag and lift coefficients.
"""
from __future__ import annotations

import math
import time

import numpy as np

import lbgpu

BYTES_PER_UPDATE = lbgpu.BYTES_PER_UPDATE


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


# ------------------------------------------------------------------------------------------
# batching
# ------------------------------------------------------------------------------------------
def batching_instances(n=512, seed=20260101):
    """Channels with nx ~ U{64..2048 step 32}, ny ~ U{32..512 step 32}, Re ~ U[20, 200],
    uMax ~ U[0.01, 0.04], radius ny/10 * U[0.8, 1.2], centre (nx/5, ny/2) * U[0.9, 1.1]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = 32 * int(rng.integers(2, 65))
        ny = 32 * int(rng.integers(1, 17))
        re = float(rng.uniform(20, 200))
        umax = float(rng.uniform(0.01, 0.04))
        r = max(2, int(round(ny / 10 * rng.uniform(0.8, 1.2))))
        ox = min(nx - r - 2, max(r + 2, int(round(nx / 5 * rng.uniform(0.9, 1.1))) + 1))
        oy = min(ny - r - 1, max(r + 2, int(round(ny / 2 * rng.uniform(0.9, 1.1))) + 1))
        out.append(dict(lx=nx, ly=ny, obst_x=ox, obst_y=oy, obst_r=r, umax=umax, re=re))
    return out


def _channel(q, precision, scheme, shift=None):
    lat = lbgpu.Lattice(q["lx"], q["ly"], precision, scheme)
    if precision in lbgpu.DEFAULT_SCALE:
        scales = lbgpu.DEFAULT_SCALE if shift is None else lbgpu.DEFAULT_SHIFT_SCALE
        lat.set_offset_scale(scales[precision])
    if shift is not None:
        lat.set_offset_shift(shift)
    lat.setup_cylinder(q["obst_x"], q["obst_y"], q["obst_r"], q["umax"], q["re"],
                       lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
    return lat


def tune_schemes(precision, sizes, steps=6):
    """Pull or AA per size class, timed on the median-sized lattice of each class present."""
    by_class = {}
    for lx, ly in sizes:
        by_class.setdefault(lbgpu.size_class(lx * ly), []).append((lx * ly, lx, ly))
    out = {}
    for c, members in sorted(by_class.items()):
        members.sort()
        _, lx, ly = members[len(members) // 2]
        scheme, t_pull, t_aa = lbgpu.tune_scheme(precision, lx, ly, steps)
        out[c] = {"scheme": scheme, "probe": [lx, ly], "ms_pull": round(t_pull, 4),
                  "ms_aa": round(t_aa, 4)}
    return out


def batching_study(precisions=("f32", "f16"), n=512, steps=2000, seed=20260101, tune=1):
    """tune=0 keeps the defaults (pull members, default tile shapes and launch form)."""
    insts = batching_instances(n, seed)
    nodes = sum(q["lx"] * q["ly"] for q in insts)
    res = {"instances": n, "seed": seed, "nodes": nodes, "steps": steps, "chunk": 50,
           "precisions": {}}
    for prec in precisions:
        if tune:
            schemes = tune_schemes(prec, [(q["lx"], q["ly"]) for q in insts])
        else:
            schemes = {lbgpu.size_class(q["lx"] * q["ly"]): {"scheme": "pull"} for q in insts}
        lats = [_channel(q, prec, schemes[lbgpu.size_class(q["lx"] * q["ly"])]["scheme"])
                for q in insts]
        try:
            with lbgpu.Batch(prec) as b:
                slots = [b.add(l) for l in lats]
                best = b.autotune(4) if tune else [0.0] * 6
                shapes = {c: list(b.shape(c)) for c in schemes}
                persistent = b.persistent
                threads = b.threads
                b.step(50)                     # first-step path and the graph capture
                b.synchronize()
                t0 = time.perf_counter()
                ms = b.step_timed(steps)
                wall_b = time.perf_counter() - t0
                launches = b.last_launches
                for s in slots:
                    b.remove(s)
            for l in lats:                     # the sequential loop, warmed the same way
                l.step(3)
            for l in lats:
                l.synchronize()
            t0 = time.perf_counter()
            for l in lats:
                l.step(steps)
            for l in lats:
                l.synchronize()
            wall_s = time.perf_counter() - t0
        finally:
            for l in lats:
                l.close()
        mb = nodes * steps / (ms * 1e-3) / 1e6
        mbw = nodes * steps / wall_b / 1e6
        msq = nodes * steps / wall_s / 1e6
        res["precisions"][prec] = {
            "batched_mlups": round(mb, 1), "batched_mlups_wall": round(mbw, 1),
            "batched_kernel_launches": launches,
            "sequential_mlups_wall": round(msq, 1), "speedup_wall": round(mbw / msq, 2),
            "batched_gbs_algorithmic": round(mb * 1e6 * BYTES_PER_UPDATE[prec] / 1e9, 1),
            "schemes": {str(k): v for k, v in schemes.items()},
            "tile_shapes": {str(k): v for k, v in shapes.items()},
            "persistent": persistent, "threads_per_tile": threads,
            "autotune_best_ms": [round(x, 4) for x in best]}
    return res


def member_shape_cases(total=16384 * 4096):
    """(label, lx, ly, members) of the shapes study: members of total / 1, 16, 256, 1024 nodes
    with lx = 4 ly, then 256 members of total / 256 nodes from 16:1 wide to 1:4 tall."""
    cases = [("alone", 16384, 4096, 1)]
    for lx, ly in ((16384, 4096), (4096, 1024), (1024, 256), (512, 128)):
        cases.append(("size", lx, ly, max(1, total // (lx * ly))))
    for lx, ly in ((4096, 64), (1024, 256), (512, 512), (256, 1024)):
        cases.append(("shape", lx, ly, max(1, total // (lx * ly))))
    return cases


def shape_obstacle(lx, ly):
    """Obstacle (x, y, r) of a shapes-study member: the benchmark's placement, with the radius
    taken from the shorter side so that narrow members keep it clear of the inlet."""
    return lx // 5 + 1, ly // 2 + 1, max(2, min(lx, ly) // 10 + 1)


def member_shape_study(precision="f16", steps=100, passes=4, total=16384 * 4096):
    """Device-timed MLUPS (best of three timings of `steps` steps after 50 warm-up steps) of each
    case of member_shape_cases; 16-bit members run in quad tiles of 128 x 4, FP32/FP64 members
    in the batch's default tiles; strips of `passes` tiles."""
    def make(lx, ly):
        lat = lbgpu.Lattice(lx, ly, precision, "pull")
        if precision in lbgpu.DEFAULT_SCALE:
            lat.set_offset_scale(lbgpu.DEFAULT_SCALE[precision])
        ox, oy, r = shape_obstacle(lx, ly)
        lat.setup_cylinder(ox, oy, r, 0.02, 100.0, lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
        return lat

    out = []
    for label, lx, ly, n in member_shape_cases(total):
        rec = {"case": label, "lx": lx, "ly": ly, "members": n,
               "perimeter_share": round((2 * lx + 2 * ly - 4) / (lx * ly), 5)}
        lats = []
        try:
            if label == "alone":
                lats.append(make(lx, ly))
                lats[0].step(20)
                lats[0].synchronize()
                ms = min(lats[0].step_timed(steps) for _ in range(3))
            else:
                lats = [make(lx, ly) for _ in range(n)]
                with lbgpu.Batch(precision) as b:
                    for c in range(6):
                        if precision in ("f16", "bf16"):
                            b.set_shape(c, 128, 4)
                        b.set_passes(c, passes)
                    for l in lats:
                        b.add(l)
                    b.step(50)
                    b.synchronize()
                    ms = min(b.step_timed(steps) for _ in range(3))
        finally:
            for l in lats:
                l.close()
        rec["mlups"] = round(n * lx * ly * steps / (ms * 1e-3) / 1e6, 1)
        rec["gbs_algorithmic"] = round(rec["mlups"] * 1e6 * BYTES_PER_UPDATE[precision] / 1e9, 1)
        out.append(rec)
        _progress(f"shapes {label} {n} x {lx}x{ly}", rec)
    return {"precision": precision, "steps": steps, "passes": passes, "nodes": total, "cases": out}


# ------------------------------------------------------------------------------------------
# serving
# ------------------------------------------------------------------------------------------
OMEGA_MAX = 1.9      # serving: uMax per request keeps omega = 1/(3 nu + 1/2) at or below this
UMAX_RANGE = (0.02, 0.1)


def serving_umax(re, r, omega_max=OMEGA_MAX, lo=UMAX_RANGE[0], hi=UMAX_RANGE[1]):
    """Peak inflow velocity of a request: 0.02, raised where the channel's viscosity
    nu = uMax 2r / Re would put omega above omega_max (small grids at high Re), capped at 0.1
    (Mach 0.17).  Requests that need more than the cap are under-resolved on their grid."""
    nu_min = (1.0 / omega_max - 0.5) / 3.0
    return float(min(hi, max(lo, nu_min * re / (2.0 * r))))


def serving_requests(n, seed=20260102, nmin=1e4, nmax=2e7, max_steps=5000, tol=1e-7,
                     umax=None):
    """Node counts log-uniform on [nmin, nmax], aspect nx/ny ~ U[2, 8], Re ~ U[20, 500];
    obstacle at (nx/5 + 1, ny/2 + 1), radius ny/10 + 1; uMax per request (serving_umax) unless
    given; arrival times are set later."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        aspect = rng.uniform(2, 8)
        ny = max(16, int(round(math.sqrt(N / aspect))))
        nx = max(32, int(round(N / ny)))
        r = ny // 10 + 1
        re = float(rng.uniform(20, 500))
        out.append(dict(lx=nx, ly=ny, obst_x=nx // 5 + 1, obst_y=ny // 2 + 1, obst_r=r,
                        umax=serving_umax(re, r) if umax is None else umax, re=re,
                        max_steps=max_steps, tol=tol, arrival=0.0, want_fields=False))
    return out


def _serve(prec, reqs, batched, budget, schemes=None, shapes=None, sample=(), shift=False, rs=False,
           solo_nodes=None):
    half = prec in lbgpu.DEFAULT_SCALE
    with lbgpu.Server(prec, budget, 100, shift=shift and half, stochastic=rs and half) as srv:
        for c, s in (schemes or {}).items():
            srv.set_scheme(c, s)
        for c, (w, npt) in (shapes or {}).items():
            srv.set_shape(c, w, npt)
        if solo_nodes is not None:
            srv.set_solo_nodes(solo_nodes)
        for k, q in enumerate(reqs):
            srv.submit(**dict(q, want_fields=k in sample))
        srv.run(batched)
        res = [srv.result(k, fields=k in sample) for k in range(len(reqs))]
        st = srv.stats()
    lat = [r["finish"] - r["arrival"] for r in res]
    ok = [r for r in res if r["converged"] != -1]
    useful = sum(r["steps"] * r["nodes"] for r in ok)
    lat_ok = [r["finish"] - r["arrival"] for r in ok]
    return {"makespan_s": round(st["makespan_s"], 3),
            "mlups": round(st["lattice_updates"] / st["makespan_s"] / 1e6, 1),
            "mlups_not_diverged": round(useful / st["makespan_s"] / 1e6, 1),
            "p50_latency_s": round(_pct(lat, 50), 4), "p99_latency_s": round(_pct(lat, 99), 4),
            "p50_latency_not_diverged_s": round(_pct(lat_ok, 50), 4),
            "p99_latency_not_diverged_s": round(_pct(lat_ok, 99), 4),
            "mean_latency_s": round(float(np.mean(lat)), 4),
            "peak_resident": st["peak_resident"], "peak_gb": round(st["peak_bytes"] / 1e9, 2),
            "converged": sum(1 for r in res if r["converged"] == 1),
            "diverged": sum(1 for r in res if r["converged"] == -1)}, res


def _progress(tag, obj):
    """One JSON line per finished part on stderr, so a long study's parts survive its end."""
    import json
    import sys
    print(json.dumps({"part": tag, **obj}), file=sys.stderr, flush=True)


def serving_study(precisions=("f32", "f16"), n=5000, seed=20260102, budget_gb=150.0,
                  load=0.95, sample_every=50, shift=0, rs=0, calib=400, plain_every=10,
                  solo_nodes=-1):
    """The request stream at the configuration's size.  Per storage type: the batched capacity
    is calibrated on the first `calib` requests present at t = 0; Poisson arrivals at `load`
    times that rate are then served batched and sequentially (plain solves one at a time, the
    same storage), the same stream for both.  A 2 % sample (every `sample_every`-th request) is
    re-run alone in FP64 for the velocity error; sequential FP64 plain solves of every
    `plain_every`-th request give the FP64 plain rate (plain_every=0 skips them; precisions=none
    runs them alone, so the parts fit separate runs).  shift=1: 16-bit requests store offsets
    from their inflow profile; rs=1: they round stochastically.  solo_nodes >= 0 overrides the
    server's size above which a request steps on its own (0: every request in the batch)."""
    reqs = serving_requests(n, seed)
    work = [q["lx"] * q["ly"] * q["max_steps"] for q in reqs]
    budget = int(budget_gb * 1e9)
    sample = set(range(0, n, sample_every))
    solo = None if solo_nodes < 0 else solo_nodes
    out = {"requests": n, "seed": seed, "budget_gb": budget_gb, "offered_load": load,
           "row_shift": bool(shift), "stochastic_rounding": bool(rs),
           "nodes_log_uniform": [1e4, 2e7], "max_steps": 5000, "tol": 1e-7,
           "umax": f"0.02, raised to keep omega <= {OMEGA_MAX} (at most {UMAX_RANGE[1]})",
           "requests_at_umax_cap": sum(1 for q in reqs if q["umax"] >= UMAX_RANGE[1]),
           "total_nodes": int(sum(q["lx"] * q["ly"] for q in reqs)),
           "fp64_sample": len(sample), "precisions": {}}
    rng = np.random.default_rng(seed + 1)
    mean_work = float(np.mean(work))
    precisions = tuple(p for p in precisions if p != "none")
    for prec in precisions:
        schemes = {c: v["scheme"] for c, v in
                   tune_schemes(prec, [(q["lx"], q["ly"]) for q in reqs]).items()}
        head = reqs[:calib]
        closed, _ = _serve(prec, head, True, budget, schemes, shift=shift, rs=rs, solo_nodes=solo)
        _progress(f"{prec} calibration", closed)
        rate = load * closed["mlups"] * 1e6 / mean_work            # requests per second
        t = np.cumsum(rng.exponential(1.0 / rate, n))
        stream = [dict(q, arrival=float(t[k] - t[0])) for k, q in enumerate(reqs)]
        served, res = _serve(prec, stream, True, budget, schemes, sample=sample, shift=shift, rs=rs,
                             solo_nodes=solo)
        _progress(f"{prec} stream batched", served)
        seq, _ = _serve(prec, stream, False, budget, shift=shift, rs=rs)
        _progress(f"{prec} stream sequential", seq)
        errs, detail = [], []
        for k in sorted(sample):
            q = reqs[k]
            if res[k]["converged"] == -1:
                detail.append({"id": k, "nodes": q["lx"] * q["ly"], "re": round(q["re"], 1),
                               "umax": round(q["umax"], 4), "diverged": True})
                continue
            with _channel(q, "f64", "pull") as lat:
                lat.step(res[k]["steps"])
                _, ux, uy = lat.macros()
            du = np.hypot(res[k]["ux"] - ux, res[k]["uy"] - uy)
            errs.append(float(np.linalg.norm(du) / max(np.linalg.norm(np.hypot(ux, uy)), 1e-300)))
            detail.append({"id": k, "nodes": q["lx"] * q["ly"], "re": round(q["re"], 1),
                           "umax": round(q["umax"], 4), "steps": res[k]["steps"], "err": errs[-1]})
        capped = [d["err"] for d in detail if "err" in d and d["umax"] >= UMAX_RANGE[1]]
        below = [d["err"] for d in detail if "err" in d and d["umax"] < UMAX_RANGE[1]]
        out["precisions"][prec] = {
            "schemes": {str(k): v for k, v in schemes.items()},
            "calibration_closed_batched": dict(closed, requests=calib),
            "arrival_rate_per_s": round(rate, 4),
            "stream_batched": served, "stream_sequential": seq,
            "throughput_ratio_same_storage": round(served["mlups_not_diverged"] /
                                                   max(seq["mlups_not_diverged"], 1e-9), 2),
            "velocity_rel_l2_vs_fp64": {"max": max(errs) if errs else None,
                                        "median": float(np.median(errs)) if errs else None,
                                        "p90": _pct(errs, 90), "n": len(errs),
                                        "below_umax_cap": {"n": len(below), "median": _pct(below, 50),
                                                           "p90": _pct(below, 90),
                                                           "max": max(below) if below else None},
                                        "at_umax_cap": {"n": len(capped), "median": _pct(capped, 50),
                                                        "max": max(capped) if capped else None},
                                        "requests": detail}}
        _progress(f"{prec} result", out["precisions"][prec])
    # sequential plain FP64 solves of every plain_every-th request, all present at t = 0
    if plain_every:
        sub = reqs[::plain_every]
        plain, _ = _serve("f64", sub, False, budget)
        _progress("f64 plain", plain)
        out["sequential_f64_plain"] = dict(plain, requests=len(sub))
        for prec in precisions:
            p = out["precisions"][prec]
            p["throughput_ratio_vs_f64_plain"] = round(p["stream_batched"]["mlups_not_diverged"] /
                                                       max(plain["mlups_not_diverged"], 1e-9), 2)
    return out


# ------------------------------------------------------------------------------------------
# precision
# ------------------------------------------------------------------------------------------
def _run_averaged(nx, ny, prec, umax, re, steps, avg_every, moment_every):
    ox, oy, r = nx // 5 + 1, ny // 2 + 1, ny // 10 + 1
    with lbgpu.Lattice(nx, ny, lbgpu.storage_form(prec)[0], "pull") as lat:
        lbgpu.configure_storage(lat, prec, umax, seed=20260101)
        lat.setup_cylinder(ox, oy, r, umax, re, lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
        m0 = lat.moments()
        half = steps // 2
        ms = lat.step_timed(half)
        fx, fy = [], []
        done = half
        while done < steps:
            k = min(avg_every, steps - done)
            ms += lat.step_timed(k)
            done += k
            lat.velocity_accumulate()
            if done % moment_every == 0:
                m = lat.moments()
                fx.append(m[3])
                fy.append(m[4])
        m1 = lat.moments()
        ux, uy, nsamp = lat.velocity_average()
    u_mean = 2.0 / 3.0 * umax                 # mean of the Poiseuille inflow profile
    dyn = 0.5 * 1.0 * u_mean ** 2 * (2 * r)
    return {"ux": ux, "uy": uy, "samples": nsamp, "mass0": m0[0], "mass1": m1[0],
            "non_finite": int(m1[6]), "cd": float(np.mean(fx)) / dyn, "cl": float(np.mean(fy)) / dyn,
            "cl_rms": float(np.sqrt(np.mean(np.square(fy)))) / dyn,
            "mlups": nx * ny * steps / (ms * 1e-3) / 1e6}


def precision_study(nx=16384, ny=4096, steps=20000, cases=((100.0, 0.02), (1000.0, 0.05)),
                    precisions=("f16", "bf16", "f16s", "bf16s", "f16r", "bf16r", "f16sr", "bf16sr"),
                    avg_every=10, moment_every=100):
    out = {"nx": nx, "ny": ny, "steps": steps, "average": f"every {avg_every} steps over the "
           f"second half", "forces": f"momentum exchange every {moment_every} steps over the "
           "second half; C = F / (0.5 rho U^2 D), U = 2/3 uMax, D = 2r", "cases": []}
    for re, umax in cases:
        ref = _run_averaged(nx, ny, "f64", umax, re, steps, avg_every, moment_every)
        nref = float(np.sqrt(np.sum(ref["ux"] ** 2 + ref["uy"] ** 2)))
        case = {"re": re, "umax": umax,
                "f64": {"mlups": round(ref["mlups"], 1), "cd": ref["cd"], "cl": ref["cl"],
                        "cl_rms": ref["cl_rms"],
                        "mass_drift": (ref["mass1"] - ref["mass0"]) / ref["mass0"],
                        "non_finite": ref["non_finite"]}}
        for prec in precisions:
            r = _run_averaged(nx, ny, prec, umax, re, steps, avg_every, moment_every)
            err = float(np.sqrt(np.sum((r["ux"] - ref["ux"]) ** 2 + (r["uy"] - ref["uy"]) ** 2))) / nref
            case[prec] = {"mlups": round(r["mlups"], 1), "vel_rel_l2_time_avg": err,
                          "mass_drift": (r["mass1"] - r["mass0"]) / r["mass0"],
                          "cd": r["cd"], "cl": r["cl"], "cl_rms": r["cl_rms"],
                          "cd_rel_err": abs(r["cd"] - ref["cd"]) / abs(ref["cd"]),
                          "cl_abs_err": abs(r["cl"] - ref["cl"]),
                          "non_finite": r["non_finite"],
                          "scale_log2": (lbgpu.DEFAULT_SHIFT_SCALE if lbgpu.storage_form(prec)[1]
                                         else lbgpu.DEFAULT_SCALE)[lbgpu.storage_form(prec)[0]],
                          "offsets_from": {"s": "Poiseuille-profile equilibrium per row",
                                           "b": f"Poiseuille-profile equilibrium per band of "
                                                f"{lbgpu.SHIFT_BAND} rows",
                                           "": "w_i"}[lbgpu.storage_form(prec)[1]],
                          "rounding": "stochastic" if lbgpu.storage_form(prec)[2] else "nearest"}
            del r
        out["cases"].append(case)
        del ref
    return out
