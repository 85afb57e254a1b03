"""Benchmark of the acPulse_vcLBM hot path on B200.

Workload (default): the operator/scheme sweep configuration -- a quasi-2D
Gaussian pulse on 1024 x 512 x 3 coarse nodes, periodic in y and z, LODI
non-reflecting faces in x, the right half (x >= 512) refined 2:1 with the
standard overlap scheme and arithmetic-average (LAG) restriction, HRR
collision (sigma = 0.98, order 3), nu = 1e-4 lattice units, eps = 1e-3,
b = 24 coarse cells.  Inputs are synthetic (seeded pulse parameters); there
is no dataset.

A step is one coarse time step (a coarse step and two fine sub-steps with the
couplings).  MLUPS = (live coarse nodes + 2 x fine nodes) x steps / s / 1e6.
`value` is the FP32-deviation form's MLUPS with the state resident in HBM;
the FP64 form runs the same steps and its MLUPS, the FP32/FP64 ratio and the
FP32 form's pressure error against FP64 are reported beside it.  Timing: CUDA events on the stream the engine
launches on, W warm-up steps, K timed steps, max over ranks.  The working set
(populations, two arrays) is larger than the 126 MB L2, so no flush is needed.

`--impl reference` times the CPU FP64 oracle (the restated reference, all
host threads) on the same workload and prints the same JSON line shape.

Two further modes reproduce the measurements behind the committed profiles
and results (they print their own lines, not the bench JSON):

  --profile   run --steps coarse steps of one case of the workload (flags
              --op --storage --order --nx --ny --nz --levels --filter
              --coupling; --batched N: the seeded batched cases in one batch
              instead), for ncu; --timed N adds N steps kernel by kernel with
              CUDA events and prints each kernel kind's device time
  --study S   sweep: the operator and scheme sweep (1024 x 512 x 3, right half
              refined, every operator x {STD, DC1} x {LAG, TOU} x nu in
              {1e-5, 1e-4, 1e-3}, 3200 steps, reflection coefficient, FP32 errors
              at nu = 1e-4); precision: the 256^3 precision form (HRR, centred
              128^3-cell patch, transverse LODI, eps in {1e-2, 1e-4}, FP32 and
              FP16 against FP64); convergence: the reflection coefficient of the
              reference-sized pulse scaled to b = 6, 12, 24, 48 cells; --out
              writes the JSON

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
       python bench.py --profile [--levels 1|2] [--op OP] [--storage S] [--steps K] [--timed N]
       python bench.py --study sweep|precision|convergence [--steps K] [--out file.json]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from acpulse_vclbm_b200 import analysis  # noqa: E402  (pure Python; loads no library)
from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case  # noqa: E402

METRIC = "MLUPS & %HBM peak: FP32-shifted vs FP64 at ≤1e-5 rel err; p99 solve latency"
E2E_SAMPLES = 3  # end-to-end solves timed; the median is reported


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--op", default="HRR")
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=3)
    ap.add_argument("--nu", type=float, default=1e-4)
    ap.add_argument("--levels", type=int, default=2, choices=[1, 2])
    ap.add_argument("--filter", default="LAG")
    ap.add_argument("--coupling", default="STD", choices=["STD", "DC1", "DC2"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched-cases", type=int, default=64, help="cases of the batched form (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=16, help="requests of the serving form (0: skip)")
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--precision-form", type=int, default=1, help="time the 256^3 precision form (0: skip)")
    ap.add_argument("--storage", default="FP32-DEV")
    ap.add_argument("--profile", action="store_true", help="profiling run of one case (see the module docstring)")
    ap.add_argument("--timed", type=int, default=0, help="--profile: N steps kernel by kernel with CUDA events")
    ap.add_argument("--batched", type=int, default=0, help="--profile: N seeded batched cases in one batch")
    ap.add_argument("--study", default="", choices=["", "sweep", "precision", "convergence"])
    ap.add_argument("--out", default="")
    return ap.parse_args()


def workload(args, storage):
    from acpulse_vclbm_b200.capi import lattice_units_case
    d = lattice_units_case(args.nx, args.ny, args.nz, op=args.op, nu_lu=args.nu, order=args.order,
                           periodic=(False, True, True), eps=1e-3, b=24.0,
                           center=(args.nx / 4.0, args.ny / 2.0, 1.0), storage=storage)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    if args.levels == 2:
        from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX
        d.max_level = 1
        d.layout = LAYOUT_BOX
        d.box_lo[:] = [args.nx // 2, 0, 0]
        d.box_hi[:] = [args.nx - 1, args.ny - 1, args.nz - 1]
        d.f2c_filter = F2C_FILTER[args.filter]
        if args.coupling != "STD":
            from acpulse_vclbm_b200.capi import C2F_REPLACE, COUPLING, F2C_REPLACE
            d.coupling = COUPLING[args.coupling]
            d.overlap = 0
            d.c2f_replace = C2F_REPLACE["Mf"]
            d.f2c_replace = F2C_REPLACE["Mc"]
    return d


def updates_per_step(desc):
    """live coarse nodes + 2 x fine nodes of one coarse step"""
    if desc.max_level == 0:
        return desc.nx * desc.ny * desc.nz
    nx, ny, nz = desc.nx, desc.ny, desc.nz
    coarse = (desc.box_lo[0] + 1 + desc.overlap) * ny * nz
    fine = (2 * (desc.box_hi[0] - desc.box_lo[0]) + 1) * 2 * ny * 2 * nz
    return coarse + 2 * fine


def config_of(args):
    scheme = "overlap 1" if args.coupling == "STD" else f"direct coupling {args.coupling}"
    lv = (f"right half (x >= {args.nx // 2}) refined 2:1, {scheme}, {args.filter} restriction"
          if args.levels == 2 else "single level")
    return {"workload": f"quasi-2D Gaussian pulse, {args.nx}x{args.ny}x{args.nz} coarse nodes, {lv}, "
                        f"periodic y/z, LODI x faces, {args.op} order 3, nu={args.nu:g} lu, eps=1e-3, b=24",
            "updates_per_step": updates_per_step(workload(args, "FP64")), "op": args.op, "levels": args.levels,
            "l2_flush": "not needed: population arrays exceed the 126 MB L2",
            "parallelism": f"replicas x{args.gpus}"}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([v.strip() for v in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key):
    """DRAM bytes per launch of the collide kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        j = json.load(open(p))
        return j.get(kernel_key)
    return None


def dist_setup(n):
    """replicas, one rank per GPU (NCCL); no lattice data crosses ranks"""
    if n <= 1:
        return None, 0
    from acpulse_vclbm_b200 import replicas
    dist, rank, _ = replicas.init("nccl", timeout_s=120)
    return dist, rank


def time_gpu(L, steps, warmup, torch, stream):
    L.step(warmup)
    L.sync()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record(stream)
    L.step(steps)
    e.record(stream)
    torch.cuda.synchronize()
    L.sync()
    return s.elapsed_time(e)


def cpu_oracle_mlups(desc, budget_s=12.0, max_steps=40, threads=0):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(desc, threads=threads)
    o.init()
    o.step(1)  # warm
    n = 0
    t0 = time.perf_counter()
    while n < max_steps and time.perf_counter() - t0 < budget_s:
        o.step(1)
        n += 1
    dt = time.perf_counter() - t0
    return updates_per_step(desc) * n / dt / 1e6, n, dt


def run_reference(args):
    dist, rank = dist_setup(args.gpus)
    if rank != 0:
        return
    d = workload(args, "FP64")
    threads = os.cpu_count() or 1
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=threads)
    o.init()
    o.step(min(args.warmup, 1))
    # each step is a bounded sample: stop after K steps or 120 s of CPU work
    n = 0
    t0 = time.perf_counter()
    while n < args.steps and time.perf_counter() - t0 < 120.0:
        o.step(1)
        n += 1
    dt = time.perf_counter() - t0
    v = updates_per_step(d) * n / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": n, "warmup": args.warmup, "ms_per_step": dt * 1e3 / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(args),
            "cpu_baseline": {"value": round(v, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": f"{n} coarse steps of the full workload in {dt:.1f} s, FP64 CPU oracle "
                                       f"(restated reference, OpenMP)"},
            "e2e": {"value": round(v, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _batched_form(args, engine, torch, device, storage, dist, rank, world):
    """One storage form of the batched configuration on this rank's share of
    the seeded cases (largest-first assignment over the ranks): the batch
    tuned, then K steps timed (max over ranks), then the same cases stepped
    one after the other for comparison."""
    from acpulse_vclbm_b200 import replicas, shard, workloads
    descs_all = workloads.batched_cases(seed=2024, n=args.batched_cases, storage=storage)
    assign = shard.assign_cases([shard.case_updates(d) for d in descs_all], world)
    _, descs = shard.my_share(descs_all, assign, rank)
    Ls = [engine.Lattice(d, device=device).init() for d in descs]
    B = engine.Batch(Ls) if Ls else None
    report = B.tune(trial_steps=3) if B else ""
    info = B.info() if B else {"groups": 0, "launches_per_step": 0, "updates_per_step": 0}
    steps = max(20, args.steps // 2)
    if B:
        B.step(3)
        B.sync()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    if B:
        B.step(steps)
        B.sync()
    batched_s = (time.perf_counter() - t0) / steps
    if B:
        B.close()
    # the same cases stepped one by one (each its own CUDA graph), for comparison
    n1 = 10
    for L in Ls:
        L.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for L in Ls:
        L.step(n1)
    for L in Ls:
        L.sync()
    alone_s = (time.perf_counter() - t0) / n1
    for L in Ls:
        L.close()
    batched_s, alone_s = replicas.reduce([batched_s, alone_s], dist, "max", device="cuda")
    upd = replicas.reduce([float(info["updates_per_step"])], dist, "sum", device="cuda")[0]
    return {"updates_per_step": int(upd), "mlups": round(upd / batched_s / 1e6, 1), "ms_per_step": batched_s * 1e3,
            "groups_rank0": info["groups"], "launches_per_step_rank0": info["launches_per_step"],
            "alone_sequential_mlups": round(upd / alone_s / 1e6, 1),
            "speedup_over_sequential": round(alone_s / batched_s, 2),
            "tuner_rank0": report.strip().split("\n")[-1] if report else None}


def bench_batched(args, engine, torch, device, peak, dist=None, rank=0, world=1):
    """The batched form: 64 seeded quasi-2D cases of uneven sizes and
    operators, one CUDA graph per coarse step, schedule chosen by the
    autotuner, in FP32 deviation and in FP64 storage; with N ranks the cases
    are sharded over the GPUs (largest-first), each rank one batch of its
    share, and the rates are whole-job (summed updates over the slowest
    rank's time)."""
    out = {"cases": args.batched_cases, "seed": 2024, "ranks": world,
           "timing": "host clock around synchronised graph launches (K steps, max over ranks)"}
    for storage, key, b in (("FP32-DEV", "fp32", 152), ("FP64", "fp64", 304)):
        r = _batched_form(args, engine, torch, device, storage, dist, rank, world)
        achieved = r["updates_per_step"] * b / (r["ms_per_step"] * 1e-3) / 1e9
        r["achieved_gbs_whole_step"] = round(achieved, 1)
        r["hbm_frac_whole_step"] = round(achieved / peak, 4)
        out[key] = r
    out["fp32_over_fp64"] = round(out["fp32"]["mlups"] / out["fp64"]["mlups"], 3)
    return out


def bench_precision(args, engine, torch, device, peak):
    """The precision form, device-timed: a 3-D pulse in a 256^3 coarse box
    with a centred 128^3-cell patch refined 2:1, HRR (sigma 0.98), nu = 1e-4,
    eps = 1e-2, b = 12, transverse LODI on all six faces; FP64, FP32 deviation
    and FP16-scaled storage on the same inputs.  K steps timed with CUDA
    events after W warm-up steps; the collide kernels' device time per step
    gives the roofline; each reduced form's pressure error is taken against
    the FP64 form after the same steps (coarse nodes the patch covers left
    out)."""
    import ctypes as C
    stream = torch.cuda.Stream()
    out = {"workload": ("3-D pulse, 256^3 coarse nodes, centred 128^3-cell patch refined 2:1, HRR order 3, "
                        "sigma 0.98, nu=1e-4 lu, eps=1e-2, b=12, transverse LODI on six faces"),
           "steps": args.steps, "warmup": args.warmup}
    ref = None
    n = 256
    lo = n // 4
    for storage, key, b in (("FP64", "fp64", 304), ("FP32-DEV", "fp32", 152), ("FP16-DEV", "fp16", 76)):
        d = study_precision_case(1e-2, storage, n)
        L = engine.Lattice(d, device=device)
        engine.lib().acp_set_stream(L._h, stream.cuda_stream)
        L.init()
        ms = time_gpu(L, args.steps, args.warmup, torch, stream)
        c, f = L.active_updates()
        upd = c + 2 * f
        km = (C.c_double * 5)()
        engine.lib().acp_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        engine.lib().acp_step_timed(L._h, 10, C.cast(km, C.c_void_p))
        achieved = upd * b / (km[1] * 1e-3) / 1e9
        row = {"mlups": round(upd * args.steps / (ms * 1e-3) / 1e6, 1), "ms_per_step": ms / args.steps,
               "updates_per_step": upd, "collide_ms_per_step": km[1], "lodi_ms_per_step": km[2],
               "coupling_ms_per_step": km[3],
               "roofline": {"achieved_gbs": round(achieved, 1), "frac": round(achieved / peak, 4),
                            "algorithmic_bytes_per_node": b}}
        p = [L.field(4, l) for l in range(2)]
        if ref is None:
            ref = (p, d.ic_eps * d.density * d.speed_of_sound ** 2)
        else:
            live = np.ones(p[0].shape, dtype=bool)
            live[lo + 1:lo + n // 2, lo + 1:lo + n // 2, lo + 1:lo + n // 2] = False
            err = max(np.abs(p[0] - ref[0][0])[live].max(), np.abs(p[1] - ref[0][1]).max()) / ref[1]
            row["pressure_err_rel_amplitude_vs_fp64"] = float(err)
        L.close()
        out[key] = row
    return out


def _serve_once(args, engine, device, base, scale, dist, rank, world):
    """serve the seeded stream with its arrival times scaled by `scale` (0:
    every request at once); requests routed over the ranks; per-request
    results gathered, whole-job rates over the slowest rank's wall time"""
    from acpulse_vclbm_b200 import replicas, serve, shard
    reqs = [serve.Request(k, t * scale, d, n) for k, (t, d, n) in enumerate(base)]
    route = shard.route_requests(reqs, world)
    _, mine = shard.my_share(reqs, route, rank)
    srv = serve.Server(budget_bytes=120 << 30, tick_steps=50, device=device)
    rep = srv.run(mine) if mine else {"wall_s": 0.0, "batch_rebuilds": 0, "ticks": 0}
    local = {r.rid: (r.latency, r.updates, r.storage) for r in srv.results}
    allres = shard.gather_results(local, dist)
    wall = replicas.reduce([rep["wall_s"]], dist, "max", device="cuda")[0]

    def stats(rows):
        lat = np.array([x[0] for x in rows])
        upd = sum(x[1] for x in rows)
        return {"requests": len(rows), "solves_per_s": round(len(rows) / wall, 3),
                "aggregate_mlups": round(upd / wall / 1e6, 1),
                "latency_p50_s": round(float(np.percentile(lat, 50)), 4) if len(lat) else None,
                "latency_p99_s": round(float(np.percentile(lat, 99)), 4) if len(lat) else None}
    rows = list(allres.values())
    out = stats(rows)
    out.update({"wall_s": round(wall, 3), "batch_rebuilds_rank0": rep["batch_rebuilds"],
                "fp32": stats([x for x in rows if x[2] == 1]), "fp64": stats([x for x in rows if x[2] == 0])})
    return out


def bench_serving(args, engine, device, dist=None, rank=0, world=1):
    """The serving form: a seeded Poisson stream of 3-D pulse solves (64^3 to
    256^3 coarse boxes with a centred 2:1 patch, 200-2000 coarse steps, five
    operators, FP32 deviation and FP64 alternating) under continuous batching
    with a 120 GB budget per GPU.  Capacity is measured with every request
    arriving at once; the same stream is then offered at 50, 80 and 95 % of
    that capacity (arrival times scaled)."""
    from acpulse_vclbm_b200 import workloads
    base = workloads.request_stream(seed=7, n=args.serve_requests, rate_hz=1.0, size_range=(64, 256),
                                    steps_range=(200, 2000))
    cap = _serve_once(args, engine, device, base, 0.0, dist, rank, world)
    capacity = cap["solves_per_s"]
    out = {"stream": (f"{len(base)} requests (seed 7), 3-D boxes 64^3-256^3 with a centred 2:1 patch, "
                      "200-2000 coarse steps, FP32-DEV / FP64 alternating, 5 operators"),
           "ranks": world, "capacity": cap, "loads": []}
    for frac in (0.5, 0.8, 0.95):
        rate = frac * capacity  # requests per second offered to the whole job
        r = _serve_once(args, engine, device, base, 1.0 / rate, dist, rank, world)
        r["offered_load"] = frac
        r["offered_rate_per_s"] = round(rate, 3)
        out["loads"].append(r)
    return out


def run_engine(args):
    import torch
    dist, rank = dist_setup(args.gpus)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from acpulse_vclbm_b200 import engine
    # the engine launches on this stream; the timing events are recorded on it
    tstream = torch.cuda.Stream()
    stream = tstream.cuda_stream

    d32 = workload(args, "FP32-DEV")
    d64 = workload(args, "FP64")
    nodes = updates_per_step(d32)

    L32 = engine.Lattice(d32, device=local)
    dims = [L32.dims(l) for l in range(d32.max_level + 1)]
    engine.lib().acp_set_stream(L32._h, stream)
    L32.init()
    L64 = engine.Lattice(d64, device=local)
    engine.lib().acp_set_stream(L64._h, stream)
    L64.init()

    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ms32 = time_gpu(L32, args.steps, args.warmup, torch, tstream)
    ms64 = time_gpu(L64, args.steps, args.warmup, torch, tstream)
    clk = clocks.stop()
    if dist:
        from acpulse_vclbm_b200 import replicas
        ms32, ms64 = replicas.reduce([ms32, ms64], dist, "max", device="cuda")

    # accuracy of the FP32 deviation form against FP64 after the same steps
    cs2 = d64.speed_of_sound ** 2
    amp = d64.ic_eps * d64.density * cs2
    live_x = slice(0, d64.box_lo[0] + 2) if d64.max_level == 1 else slice(None)
    rel_err = float(np.abs(L32.field(4)[..., live_x] - L64.field(4)[..., live_x]).max() / amp)
    if d64.max_level == 1:
        rel_err = max(rel_err, float(np.abs(L32.field(4, 1) - L64.field(4, 1)).max() / amp))

    # per-kernel device time (events between launches) for the roofline
    import ctypes as C
    km = (C.c_double * 5)()
    engine.lib().acp_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    engine.lib().acp_step_timed(L32._h, 20, C.cast(km, C.c_void_p))
    collide_ms32 = km[1]
    km64 = (C.c_double * 5)()
    engine.lib().acp_step_timed(L64._h, 20, C.cast(km64, C.c_void_p))
    lps = C.c_int()
    engine.lib().acp_launches_per_step(L32._h, C.byref(lps))
    peak, peak_kind = peaks()
    alg_bytes = nodes * 2 * 19 * 4  # FP32 deviation storage: read 19 + write 19 per node update
    achieved = alg_bytes / (collide_ms32 * 1e-3) / 1e9  # collide launches of one coarse step
    L32.close()
    L64.close()

    # end to end through the C ABI with host buffers: create (H2D of node
    # classes and boundary wiring), init, K steps, D2H of the pressure field of
    # every level into the caller's page-locked host buffers (allocated
    # before the timed region, as a caller keeps its output buffers).  The
    # whole solve is timed three times and the median kept: a single sample of
    # a ~25 ms region picks up one-off host stalls of the box.
    outs = [torch.empty((nz, ny, nx), dtype=torch.float64, pin_memory=True).numpy() for nx, ny, nz in dims]
    samples = []
    for _ in range(E2E_SAMPLES):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Le = engine.Lattice(d32, device=local).init()
        Le.step(args.steps)
        Le.sync()
        for l in range(d32.max_level + 1):
            Le.field(4, l, out=outs[l])
        t1 = time.perf_counter()
        Le.close()
        samples.append(t1 - t0)
    stored = sum(a * b * c for a, b, c in dims)
    h2d = stored + 2 * (d32.ny * d32.nz) * 80  # node classes + LODI wiring records
    d2h = stored * 8  # the pressure fields (FP64, formed on the device)
    e2e_s = float(np.median(samples))
    if dist:
        from acpulse_vclbm_b200 import replicas
        e2e_s = replicas.reduce([e2e_s], dist, "max", device="cuda")[0]
    e2e = nodes * args.steps * args.gpus / e2e_s / 1e6  # every rank runs its own replica end to end

    batched = serving = precision = None
    if args.precision_form:
        precision = bench_precision(args, engine, torch, local, peak)
    if args.batched_cases > 0:
        world = args.gpus if dist else 1
        batched = bench_batched(args, engine, torch, local, peak, dist, rank, world)
    if args.serve_requests > 0:
        serving = bench_serving(args, engine, local, dist, rank, args.gpus if dist else 1)
    mlups32 = nodes * args.steps / (ms32 * 1e-3) / 1e6 * args.gpus
    mlups64 = nodes * args.steps / (ms64 * 1e-3) / 1e6 * args.gpus
    cpu = None
    if rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
        v, n, dt = cpu_oracle_mlups(d64, threads=os.cpu_count() or 1)
        cpu = {"value": round(v, 3), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{n} coarse steps of the full workload in {dt:.1f} s (FP64 CPU oracle, OpenMP)"}
    if rank == 0:
        line = {"metric": METRIC, "value": round(mlups32, 2), "unit": "MLUPS", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config_of(args),
                "fp64": {"value": round(mlups64, 2), "unit": "MLUPS", "ms_per_step": ms64 / args.steps,
                         "collide_ms": km64[1]},
                "fp32_over_fp64": round(mlups32 / mlups64, 3),
                "fp32_pressure_err_rel_amplitude": rel_err,
                "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                             "kernel": "collide+push kernels of one coarse step (FP32 deviation)",
                             "algorithmic_bytes_per_node": 152, "traffic": ncu_traffic("collide_fp32"),
                             "kernel_ms": {"moments": km[0], "collide": km[1], "lodi": km[2], "probes": km[4]}},
                "cpu_baseline": cpu,
                "e2e": {"value": round(e2e, 2), "unit": "MLUPS", "h2d_bytes_per_step": h2d // args.steps,
                        "d2h_bytes_per_step": d2h // args.steps,
                        "timing": f"median of {E2E_SAMPLES} end-to-end solves (wall clock around create, init, "
                                  f"{args.steps} steps and the pressure fields read back)",
                        "samples_ms": [round(x * 1e3, 3) for x in samples]},
                "gpu_launches": lps.value * args.steps,
                "clocks": clk,
                "precision_form": precision,
                "batched": batched,
                "serving": serving}
        print(json.dumps(line), flush=True)
    if dist:
        from acpulse_vclbm_b200 import replicas
        replicas.finish(dist)


def run_profile(args):
    """A few coarse steps of one case (or of the seeded batched cases), for
    ncu; with --timed, per-kernel-kind device times by CUDA events."""
    import ctypes as C
    from acpulse_vclbm_b200 import engine
    if args.batched:
        from acpulse_vclbm_b200 import workloads
        Ls = [engine.Lattice(d).init() for d in workloads.batched_cases(seed=2024, n=args.batched)]
        B = engine.Batch(Ls)
        B.step(args.steps)
        B.sync()
        print(B.info())
        B.close()
        for L in Ls:
            L.close()
        return
    d = workload(args, args.storage)
    L = engine.Lattice(d).init()
    L.step(args.steps)
    L.sync()
    if args.timed:
        km = (C.c_double * 5)()
        engine.lib().acp_step_timed.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        engine.lib().acp_step_timed(L._h, args.timed, C.cast(km, C.c_void_p))
        c, f = L.active_updates()
        nodes = c + 2 * f
        b = {"FP64": 8, "FP32-DEV": 4, "FP16-DEV": 2}[args.storage] * 38
        print(f"{args.op} {args.storage} order {args.order} {args.nx}x{args.ny}x{args.nz} levels {args.levels}: "
              f"collide {km[1]*1e3:.1f} us ({nodes * b / (km[1] * 1e-3) / 1e9:.0f} GB/s algorithmic), "
              f"lodi {km[2]*1e3:.1f} us, coupling {km[3]*1e3:.1f} us, updates/step {nodes}", flush=True)
    L.close()


# ---------------------------------------------------------------------------
# studies of the pulse configurations (--study), GPU, FP64 unless stated

OPS5 = ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"]


def _study_run(d, steps, probes):
    from acpulse_vclbm_b200 import engine
    L = engine.Lattice(d).init()
    L.set_probes(probes)
    L.step(steps)
    L.sync()
    s = L.probes()
    p = [L.field(4, l) for l in range(d.max_level + 1)]
    L.close()
    return s, p


def study_sweep(steps=3200, nx=1024, ny=512):
    from acpulse_vclbm_b200.engine import AcpError
    rows = []
    uni = {}
    p0 = None
    for op in OPS5:
        for nu in (1e-5, 1e-4, 1e-3):
            du = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                         center=(nx / 4.0, ny / 2.0, 1.0), refined=False)
            try:
                uni[(op, nu)], _ = _study_run(du, steps, analysis.interface_probes(du))
            except AcpError as e:
                rows.append({"op": op, "nu": nu, "uniform_error": str(e)})
                continue
            p0 = du.density * du.speed_of_sound ** 2
            for coupling in ("STD", "DC1"):
                for filt in ("LAG", "TOU"):
                    t0 = time.perf_counter()
                    d = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                                center=(nx / 4.0, ny / 2.0, 1.0), filt=filt, coupling=coupling)
                    try:
                        s64, f64 = _study_run(d, steps, analysis.interface_probes(d))
                    except AcpError as e:  # a numerical blow-up is a result of the sweep
                        row = {"op": op, "nu": nu, "coupling": coupling, "filter": filt, "R": None,
                               "error": str(e)}
                        rows.append(row)
                        print(json.dumps(row), flush=True)
                        continue
                    w = min(steps, analysis.window_steps(d))
                    r = analysis.reflection_coefficient(s64[:, 0], uni[(op, nu)][:, 0], p0, w)
                    row = {"op": op, "nu": nu, "coupling": coupling, "filter": filt, "R": r, "window_steps": w}
                    if nu == 1e-4:
                        d32 = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                                      center=(nx / 4.0, ny / 2.0, 1.0), filt=filt,
                                                      coupling=coupling, storage="FP32-DEV")
                        try:
                            s32, f32 = _study_run(d32, steps, analysis.interface_probes(d32))
                        except AcpError as e:
                            row["fp32_error"] = str(e)
                            rows.append(row)
                            continue
                        amp = d.ic_eps * d.density * d.speed_of_sound ** 2
                        live = slice(0, nx // 2 + 1 + d.overlap)
                        e = [f32[0][..., live] - f64[0][..., live], f32[1] - f64[1]]
                        n = sum(x.size for x in e)
                        row["fp32_l2_err_rel_amp"] = float(np.sqrt(sum((x ** 2).sum() for x in e) / n) / amp)
                        row["fp32_max_err_rel_amp"] = float(max(np.abs(x).max() for x in e) / amp)
                        row["fp32_probe_err_rel_amp"] = float(np.abs(s32 - s64).max() / amp)
                        # the FP32 form's R from its own pair of runs (refined and
                        # uniform, both FP32), against the FP64 pair's
                        key32 = (op, nu, "FP32-DEV")
                        if key32 not in uni:
                            du32 = analysis.interface_case(nx, ny, 3, op=op, nu=nu, eps=1e-3, b=24.0,
                                                           center=(nx / 4.0, ny / 2.0, 1.0), refined=False,
                                                           storage="FP32-DEV")
                            uni[key32], _ = _study_run(du32, steps, analysis.interface_probes(du32))
                        r32 = analysis.reflection_coefficient(s32[:, 0], uni[key32][:, 0], p0, w)
                        row["fp32_R"] = r32
                        row["fp32_R_abs_err"] = abs(r32 - r)
                        row["fp32_R_rel_err"] = abs(r32 - r) / r
                    row["seconds"] = time.perf_counter() - t0
                    rows.append(row)
                    print(json.dumps(row), flush=True)
    return {"study": "operator and scheme sweep", "nx": nx, "ny": ny, "nz": 3, "steps": steps, "rows": rows}


def study_precision_case(eps, storage, n=256):
    lo, hi = n // 4, n // 4 + n // 2
    d = lattice_units_case(n, n, n, op="HRR", nu_lu=1e-4, order=3, periodic=(False, False, False), eps=eps,
                           b=12.0, center=(n / 2.0, n / 2.0, n / 2.0), storage=storage, ic_dims=3)
    d.hybrid_sigma = 0.98
    d.transverse = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [lo, lo, lo]
    d.box_hi[:] = [hi, hi, hi]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


def study_precision(steps=300, n=256):
    rows = []
    c = n // 2
    lo = n // 4
    probes = [(1, 2 * (lo + 10), 2 * c, 2 * c), (0, lo - 10, c, c)]  # 10 cells inside and outside the patch face
    for eps in (1e-2, 1e-4):
        ref = None
        for storage in ("FP64", "FP32-DEV", "FP16-DEV"):
            d = study_precision_case(eps, storage, n)
            t0 = time.perf_counter()
            from acpulse_vclbm_b200 import engine
            L = engine.Lattice(d).init()
            L.set_probes(probes)
            L.step(steps)
            L.sync()
            ms = (time.perf_counter() - t0) * 1e3 / steps
            s = L.probes()
            f = [L.field(4, l) for l in range(2)]
            c_, fi = L.active_updates()
            L.close()
            amp = eps * d.density * d.speed_of_sound ** 2
            row = {"eps": eps, "storage": storage, "steps": steps, "ms_per_step_incl_setup": ms,
                   "updates_per_step": c_ + 2 * fi}
            if ref is None:
                ref = (s, f)
            else:
                live = np.ones(f[0].shape, dtype=bool)
                live[lo + 1:lo + n // 2, lo + 1:lo + n // 2, lo + 1:lo + n // 2] = False  # covered coarse nodes
                row["probe_err_rel_amp"] = float(np.abs(s - ref[0]).max() / amp)
                row["field_max_err_rel_amp"] = float(max(np.abs(f[0] - ref[1][0])[live].max(),
                                                         np.abs(f[1] - ref[1][1]).max()) / amp)
            rows.append(row)
            print(json.dumps(row), flush=True)
    return {"study": "precision form", "n": n, "steps": steps, "rows": rows}




def study_convergence(bs=(6.0, 12.0, 24.0, 48.0), ops=("SRT", "MRT-RM"), couplings=("STD", "DC1")):
    """Reflection coefficient of the reference-sized pulse (128 x 64 x 3, b = 6)
    scaled to b cells: grid, pulse, centre and steps times b / 6, lattice
    viscosity 1e-3 x b / 6 (a physically similar refinement), FP64; the
    observed order between successive b."""
    rows = []
    for op in ops:
        for coupling in couplings:
            prev = None
            for b in bs:
                s = b / 6.0
                nx, ny = int(128 * s), int(64 * s)
                kw = dict(op=op, nu=1e-3 * s, eps=1e-3, b=b, center=(32.0 * s, 32.0 * s, 1.0))
                d = analysis.interface_case(nx, ny, 3, coupling=coupling, **kw)
                du = analysis.interface_case(nx, ny, 3, refined=False, **kw)
                w = analysis.window_steps(d)
                s_ref, _ = _study_run(d, w, analysis.interface_probes(d)[:1])
                s_uni, _ = _study_run(du, w, analysis.interface_probes(du)[:1])
                r = analysis.reflection_coefficient(s_ref[:, 0], s_uni[:, 0], d.density * d.speed_of_sound ** 2, w)
                row = {"op": op, "coupling": coupling, "b": b, "nx": nx, "ny": ny, "steps": w, "R": r}
                if prev:
                    row["order"] = float(np.log(prev / r) / np.log(2.0))
                prev = r
                rows.append(row)
                print(json.dumps(row), flush=True)
    return {"study": "reflection coefficient under refinement", "rows": rows}

def run_study(args):
    if args.study == "sweep":
        res = study_sweep(steps=args.steps if args.steps != 200 else 3200)
    elif args.study == "precision":
        res = study_precision(steps=args.steps if args.steps != 200 else 300)
    else:
        res = study_convergence()
    if args.out:
        json.dump(res, open(args.out, "w"), indent=1)


if __name__ == "__main__":
    a = parse()
    if a.profile:
        run_profile(a)
    elif a.study:
        run_study(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_engine(a)
