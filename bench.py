#!/usr/bin/env python
"""Benchmark of the B200 hot path (the driver's bench contract).

One step = one pass of ORCTM's nonhydrostatic hot path (OCUAD, OCVAD, OCWAD,
OCADPO for T, S and a passive tracer, OCTDIFF, OCVISC, OCVTOT_NH with its
Poisson solve to a 1e-10 relative residual), orctm.f90:1454-1562, on a seeded
synthetic instance of the 1024 x 1024 x 80 configuration (c3) resident on one
GPU.  Multi-GPU runs are independent replicas (one instance per rank, weak
scaling, no collective on the data path); timing is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per interior cell per launch of each launcher group
# (each distinct array the math needs read once, each output written once;
# thickness/mask geometry is compressed to 2D and counts 0 B).
BYTES_PER_CELL_F64 = {
    "ocuad": 40, "ocvad": 40, "ocwad": 40, "ocadpo": 40,
    "ocvisc": 56, "nh_rhs": 56, "nh_post": 56,
    "pcg_spmv": 32, "pcg_col": 56, "resid": 24,
}


METRIC = "cell-steps/s (hot path incl. Poisson solve @1e-10 rel. residual)"
DATA = "synthetic (seeded PCG64, base seed 20261203; generators of the c1-c5 workloads)"


def workload_config(inst: dict) -> dict:
    """The config object of the bench line (both arms)."""
    cells = inst["nx"] * inst["ny"] * inst["nz"]
    return {"workload": f"{inst['name']} {inst['nx']}x{inst['ny']}x{inst['nz']} "
                        f"dt={inst['dt']:g}s, one instance per GPU",
            "cells_per_gpu": cells, "tracers": inst["ntracers"],
            "l2": "inputs larger than L2 (each 3D field "
                  f"{8 * cells / 1e9:.2f} GB vs 126 MB L2)",
            "solver": "FP64 PCG (line preconditioner, scaled operator) in "
                      "double-double-residual refinement"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    try:  # one rank per GPU; ranks beyond the visible GPUs share them (replicas)
        import torch

        if torch.cuda.is_available() and torch.cuda.device_count() > 0:
            local = local % torch.cuda.device_count()
    except Exception:
        pass
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend="gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def workload(args, rank, closed=False):
    from orctm_b200 import configs

    over = {"closed": True} if closed else {}
    if args.size:
        nx, ny, nz = (int(v) for v in args.size.split("x"))
        over.update({"nx": nx, "ny": ny, "nz": nz})
    t = time.time()
    inst = configs.make_instance(args.config, index=rank, **over)
    log(f"[bench] rank {rank}: instance {args.config} {inst['nx']}x{inst['ny']}x{inst['nz']} "
        f"generated in {time.time() - t:.1f}s")
    return inst


def cpu_sample(args, solver_rtol=1e-10, steps=None, warmup=1):
    """The CPU restatement (oracle) timed on the host cores on a bounded sample
    of the same workload: hot-path steps of a sub-domain generated with the
    same generators (same dx, dz, dt, bathymetry statistics).  With ``steps``
    it times exactly that many after ``warmup`` untimed ones; otherwise it
    runs for about ``args.cpu_seconds``."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    from orctm_b200 import configs

    nx, ny, nz = args.cpu_sample
    inst = configs.make_instance(args.config, builder=O.build_grid, nx=nx, ny=ny, nz=nz)
    orc = O.Oracle(inst)
    st = configs.copy_state(inst)
    for _ in range(max(warmup, 1)):  # warm-up (and warm start)
        orc.step_hotpath(st, solver="fgmres", rtol=solver_rtol)
    t0 = time.perf_counter()
    target = steps
    steps = 0
    while True:
        info = orc.step_hotpath(st, solver="fgmres", rtol=solver_rtol)
        steps += 1
        if target is not None:
            if steps >= target:
                break
        elif time.perf_counter() - t0 > args.cpu_seconds or steps >= 50:
            break
    dt_ = time.perf_counter() - t0
    cells = nx * ny * nz
    return {"value": cells * steps / dt_, "unit": "cell-steps/s",
            "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
            "sample": f"{steps} hot-path steps of a {nx}x{ny}x{nz} sub-domain with the "
                      f"{args.config} generators (C restatement, OpenMP, FGMRES(30)+line "
                      f"preconditioner to {solver_rtol:g})",
            "ms_per_step": 1e3 * dt_ / steps, "last_krylov_its": int(info["its"])}


def run_reference(args, ws, rank, pg):
    """The reference arm: the reference's Fortran/PETSc path cannot be built on
    this image, so its CPU restatement (the oracle, OpenMP on every host core)
    runs the same workload's generators on a bounded sub-domain, one hot-path
    step per bench step (W untimed, K timed).  Rank 0 only.  The line's
    config names the sub-domain it timed, and the full workload it samples."""
    if rank != 0:
        return 0
    from orctm_b200 import configs

    over = {}
    if args.size:
        nx, ny, nz = (int(v) for v in args.size.split("x"))
        over = {"nx": nx, "ny": ny, "nz": nz}
    full = configs.raw_instance(args.config, index=0, **over)
    nx, ny, nz = args.cpu_sample
    inst = configs.raw_instance(args.config, index=0, nx=nx, ny=ny, nz=nz)
    cb = cpu_sample(args, steps=args.steps, warmup=args.warmup)
    cfg = workload_config(inst)
    if (nx, ny, nz) != (full["nx"], full["ny"], full["nz"]):
        cfg["workload"] = (f"{inst['name']} {nx}x{ny}x{nz} sub-domain sample of the "
                           f"{full['nx']}x{full['ny']}x{full['nz']} workload (same generators, "
                           f"dx, dz, dt={inst['dt']:g}s)")
        cfg["sampled_workload"] = workload_config(full)["workload"]
    cfg["solver"] = "FGMRES(30) + column (line) preconditioner, FP64, C restatement"
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"],
            "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": cfg,
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def tracer_content(inst, t) -> float:
    """Sum of T * V over the wet interior cells, V = DLXP DLYP (DDPO + ZO at
    the surface level): the tracer content the advection and diffusion
    conserve apart from the fluxes through open boundaries."""
    area = (inst["dlxp"] * inst["dlyp"])[1:-1, 1:-1]
    tot = 0.0
    for k in range(inst["ke"]):
        th = inst["ddpo"][1:-1, 1:-1, k] + (inst["zo"][1:-1, 1:-1] if k == 0 else 0.0)
        tot += float(np.sum(t[1:-1, 1:-1, k] * inst["weto"][1:-1, 1:-1, k] * th * area))
    return tot


def compare_forms(inst, a, b, nsteps) -> dict:
    """Fields of the FP32-refined form (b) against the FP64 form (a) after the
    same steps from the same state: relative max-norm differences, and each
    form's tracer-content drift from the initial state."""
    def rel(x, y):
        return float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))

    out = {"steps": nsteps, "rel_maxnorm": {}, "tracer_content_drift": {}}
    for k in ("pnh", "uoo", "voe", "wno"):
        out["rel_maxnorm"][k] = rel(b.download(k), a.download(k))
    for n in range(a.ntr):
        ta, tb = a.download(f"tracer{n}"), b.download(f"tracer{n}")
        out["rel_maxnorm"][f"tracer{n}"] = rel(tb, ta)
        c0 = tracer_content(inst, inst["tracers"][n])
        ca, cb = tracer_content(inst, ta), tracer_content(inst, tb)
        out["tracer_content_drift"][f"tracer{n}"] = {
            "fp64": (ca - c0) / abs(c0), "fp32_refined": (cb - c0) / abs(c0),
            "forms_differ_by": (cb - ca) / abs(c0)}
    out["note"] = ("open W and S boundaries: the content changes through boundary fluxes; "
                   "the two forms' drifts differ by forms_differ_by")
    return out


def timed_steps(gpu, k, pg):
    from orctm_b200.api import Instance

    barrier(pg)
    gpu.synchronize()
    n0 = Instance.kernel_launches()
    gpu.timer_start()
    stats = [gpu.step_hotpath() for _ in range(k)]
    ms = gpu.timer_stop()
    launches = Instance.kernel_launches() - n0
    barrier(pg)
    return ms, stats, launches


def run_whole_step(inst, cells, args, ws, rank, pg, local, hot_ms_per_step):
    """The whole reference step on the device (orctm_step_full: OCTHER, OCWIND,
    OCTIMF, OCMODMOM, OCBARP, OCCLIT, TRONEU's 250 SOR sweeps, OCVTRO, OCVTOT,
    then the hot path) on a third instance of the same workload: only the
    solve's scalars and OCCLIT's CONTRA reach the host per step."""
    from orctm_b200 import configs, grid
    from orctm_b200.api import Instance

    if any(inst["ob"].values()):
        # the same grid with its open sides closed: the reference's explicit
        # open-boundary elevation row (troneu.f90:67-102) grows at this dt
        inst = workload(args, rank, closed=True)
    gpu = Instance(inst, device=local)
    gpu.upload_state(configs.copy_state(inst))
    gpu.set_solver("fp64", rtol=1e-10, maxit=5000)
    gpu.set_thermo(**configs.make_thermo(inst))
    cor = configs.make_coriolis(inst)
    gpu.set_coriolis(cor["ftwou"], cor["ftwov"], cor["gila"], cor["giph"], cor["omega"])
    deuto, deute = grid.uv_depths(inst["depto"])
    gpu.set_barotropic(deuto, deute, configs.barotropic_minvalue(inst))
    gpu.ocwind(**configs.make_wind(inst))
    for s in range(args.warmup):
        gpu.step_full(s + 1, check_contra=False)
    barrier(pg)
    gpu.synchronize()
    n0 = Instance.kernel_launches()
    gpu.timer_start()
    stats = [gpu.step_full(args.warmup + s + 1, check_contra=False) for s in range(args.steps)]
    ms = gpu.timer_stop()
    launches = Instance.kernel_launches() - n0
    barrier(pg)
    ms = max_over_ranks(pg, ms)
    # the hot path's share in this state (its solve takes more iterations than
    # in the headline state): per-launcher device time of the hot-path
    # kernels over a few more, untimed whole steps
    nprof = min(args.steps, 3)
    gpu.set_profiling(True)
    for s in range(nprof):
        gpu.step_full(args.warmup + args.steps + s + 1, check_contra=False)
    hot_in_whole = sum(v["ms"] for v in gpu.profile().values()) / nprof
    gpu.set_profiling(False)
    hot_in_whole = max_over_ranks(pg, hot_in_whole)
    gpu.close()
    per = ms / args.steps
    return {"value": ws * cells * args.steps / (ms / 1e3), "unit": "cell-steps/s",
            "ms_per_step": per, "hot_path_ms_per_step": hot_in_whole,
            "before_hot_path_ms_per_step": per - hot_in_whole,
            "headline_hot_path_ms_per_step": hot_ms_per_step,
            "hot_path_basis": f"sum of the hot-path launchers' CUDA-event times over {nprof} more "
                              "whole steps with per-launcher timing on (the solve's loop then "
                              "runs from the host), so the split slightly favours the hot path",
            "poisson_iterations": statistics.mean(s["iterations"] for s in stats),
            "contra_max": max(s["contra"] for s in stats),
            "steps_above_contra_limit": sum(bool(s["unstable"]) for s in stats),
            "gpu_launches_per_step": launches / args.steps,
            "boundaries": "open W and S closed (the reference's open-boundary elevation row in "
                          "TRONEU is explicit and unstable at this dt)" if inst["name"] != "c1"
                          else "closed, as the workload",
            "note": "OCTHER (EOS " + ("linear" if inst["name"] == "c1" else "UNESCO") +
                    "), OCWIND, OCTIMF, OCMODMOM, OCBARP, OCCLIT, TRONEU (250 SOR sweeps), OCVTRO, "
                    "OCVTOT and the hot path, all on the device; state resident, no host copies"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3")
    ap.add_argument("--workload", default="step", choices=["step", "c4", "c5", "obc"],
                    help="step: one instance per GPU (the headline); c4: ensemble batch vs one at "
                         "a time; c5: served requests with Poisson arrivals; obc: open-boundary "
                         "tide forcing and sponge on the tidally forced c2 box")
    ap.add_argument("--members", type=int, default=64, help="c4/c5: requests")
    ap.add_argument("--distinct", type=int, default=16,
                    help="c4/c5: distinct seeded instances the requests cycle through")
    ap.add_argument("--member-steps", type=int, default=20, help="c4/c5: steps per request")
    ap.add_argument("--slots", type=int, default=16, help="c4/c5: requests in flight")
    ap.add_argument("--rate", type=float, default=20.0, help="c5: Poisson arrival rate (1/s)")
    ap.add_argument("--size", default=None, help="override nx x ny x nz (e.g. 256x256x60)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-whole-step", action="store_true",
                    help="skip the whole-step (orctm_step_full) measurement")
    ap.add_argument("--tuning", type=lambda s: tuple(int(v) for v in s.split(",")), default=None,
                    help="COL,SPMV: pin the FP64 Poisson kernel variants instead of autotuning "
                         "(profiling a given variant)")
    ap.add_argument("--nvtx", action="store_true",
                    help="wrap the event-timed FP64 steps (every solver iteration launched "
                         "on its own) in the NVTX range fp64_steps, for an ncu launch list "
                         "(--nvtx --nvtx-include fp64_steps/)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cpu-sample", type=lambda s: tuple(int(v) for v in s.split("x")),
                    default=None, help="sub-domain the CPU restatement times (default: the "
                    "whole c1 slice; 128x128xNZ for the 3D configurations)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.cpu_sample is None:
        args.cpu_sample = {"c1": (512, 1, 60), "c2": (128, 128, 60)}.get(args.config, (128, 128, 80))
    ws, rank, local, pg = dist_setup()
    if args.impl == "reference":
        return run_reference(args, ws, rank, pg)
    if args.workload == "obc":
        return run_obc(args, ws, rank, local, pg)
    if args.workload != "step":
        return run_ensemble(args, ws, rank, local, pg)

    from orctm_b200 import configs
    from orctm_b200.api import Instance

    inst = workload(args, rank)
    cells = inst["nx"] * inst["ny"] * inst["nz"]
    gpu = Instance(inst, device=local)
    gpu.upload_state(configs.copy_state(inst))
    gpu.set_solver("fp64", rtol=1e-10, maxit=5000)
    if args.tuning:
        gpu.set_tuning(*args.tuning)
    for _ in range(args.warmup):
        gpu.step_hotpath()

    # ---- FP64 drop-in path (headline) ------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    gpu.set_profiling(True)
    if args.nvtx:
        import torch

        torch.cuda.nvtx.range_push("fp64_steps")
    ms, stats, launches = timed_steps(gpu, args.steps, pg)
    if args.nvtx:
        torch.cuda.nvtx.range_pop()
    prof = gpu.profile()
    gpu.set_profiling(False)
    ck = clocks.stop()
    # the same steps without event brackets: the timed number
    ms, stats2, launches = timed_steps(gpu, args.steps, pg)
    ms_max = max_over_ranks(pg, ms)
    value = ws * cells * args.steps / (ms_max / 1e3)
    poisson_ms = statistics.mean(s["solve_ms"] for s in stats2)
    iters = statistics.mean(s["iterations"] for s in stats2)
    relres = max(s["relres"] for s in stats2)

    # ---- FP32-refined solver form ------------------------------------------
    # a second instance from the same initial state, stepped as often as the
    # FP64 one (W warm-up, K untimed, K timed), so that the two forms' fields
    # can be compared after the same number of steps
    nsteps = args.warmup + 2 * args.steps
    gpu2 = Instance(inst, device=local)
    gpu2.upload_state(configs.copy_state(inst))
    gpu2.set_solver("fp32_refined", rtol=1e-10, maxit=5000)
    for _ in range(args.warmup + args.steps):
        gpu2.step_hotpath()
    ms_m, stats_m, _ = timed_steps(gpu2, args.steps, pg)
    ms_m = max_over_ranks(pg, ms_m)
    mixed = {"value": ws * cells * args.steps / (ms_m / 1e3), "unit": "cell-steps/s",
             "ms_per_step": ms_m / args.steps,
             "poisson_ms": statistics.mean(s["solve_ms"] for s in stats_m),
             "poisson_iterations": statistics.mean(s["iterations"] for s in stats_m),
             "outer_iterations": statistics.mean(s["outer_iterations"] for s in stats_m),
             "relres_max": max(s["relres"] for s in stats_m)}
    mixed["speedup_vs_fp64"] = mixed["value"] / value
    mixed["solver_speedup_vs_fp64"] = poisson_ms / mixed["poisson_ms"]
    mixed["vs_fp64"] = compare_forms(inst, gpu, gpu2, nsteps)
    tuning = {"fp64": list(gpu.tuning("fp64")), "fp32_refined": list(gpu2.tuning("fp32_refined")),
              "meaning": "(column-kernel variant, stencil-kernel variant) picked by the autotuner"}
    gpu2.close()

    # ---- roofline of the dominant kernel --------------------------------
    hbm, peak_kind = peaks()
    top = max((k for k in prof if prof[k]["launches"] > 0), key=lambda k: prof[k]["ms"])
    per_launch_ms = prof[top]["ms"] / prof[top]["launches"]
    # algorithmic bytes per cell x the cells of a launch; the solver kernels
    # skip the land rows among them (decoupled, exact zeros), which the
    # measured traffic shows
    wet = int(np.asarray(inst["weto"])[1:-1, 1:-1, :].sum())
    bpl = BYTES_PER_CELL_F64.get(top, 0) * cells
    achieved = bpl / (per_launch_ms / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        if top in tj:
            # measured per variant (DRAM bytes per cell of the whole grid):
            # reported only for the variant the tuner picked
            var = str(tuning["fp64"][0] if top == "pcg_col" else tuning["fp64"][1])
            per = tj[top].get("by_variant", {}).get(var)
            traffic = per * cells if per is not None else None
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind ==
                "measured" else "fallback 6.65 TB/s",
                "bytes_per_launch": bpl, "avg_launch_ms": per_launch_ms,
                "bytes_basis": "all cells (%d; of them %d wet: the solver kernels skip the "
                               "land rows' loads and stores)" % (cells, wet),
                "breakdown_ms_per_step": {k: round(v["ms"] / args.steps, 3) for k, v in prof.items()},
                "algorithmic_bytes_per_cell": BYTES_PER_CELL_F64}

    # ---- end to end through the public API with host buffers ---------------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(gpu, inst, cells, args, ws, pg)

    whole = None
    if not args.no_whole_step:
        whole = run_whole_step(inst, cells, args, ws, rank, pg, local, ms_max / args.steps)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_sample(args)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"error": repr(ex)}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA,
            "config": workload_config(inst),
            "poisson_ms": poisson_ms, "poisson_iterations": iters, "relres_max": relres,
            "mixed": mixed, "whole_step": whole, "solver_tuning": tuning, "roofline": roofline,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": ck,
        }
        print(json.dumps(line), flush=True)
    gpu.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def _band_cells(inst, obc):
    """Cells of the u-, v- and p-point (2D) sponge bands: the cells
    orctm_obc_uv / orctm_obc_eta read and write."""
    ie, je, ke = inst["ie"], inst["je"], inst["ke"]
    out = {}
    for kind, (ilo, jlo, ni, nj) in {"u": (0, 1, ie + 1, je), "v": (1, 0, ie, je + 1),
                                     "z": (1, 1, ie, je)}.items():
        I = np.arange(ni)[:, None] + ilo
        J = np.arange(nj)[None, :] + jlo
        d = [I + 1 if kind == "u" else I, ie - I + 1, J + 1 if kind == "v" else J, je - J + 1]
        on = [bool(inst["ob"][k]) and bool(obc["sponge"][b])
              for b, k in enumerate(("west", "east", "north", "south"))]
        band = np.zeros((ni, nj), dtype=bool)
        for b in range(4):
            if on[b]:
                band |= np.broadcast_to(d[b] <= obc["width"][b], (ni, nj))
        out[kind] = int(band.sum()) * (1 if kind == "z" else ke)
    return out


def run_obc(args, ws, rank, local, pg):
    """Open-boundary tide forcing + 1/x sponge (orctm_obc_uv, orctm_obc_eta;
    mo_obcs.f90) and the T/S sponge (orctm_obc_ts) on the tidally forced c2
    box (W+S open, 30-cell sponges):
    device time per call (CUDA events on the handle's stream, max over
    ranks), the band bytes it moves, and its share of a hot-path step.  The
    velocity call is timed with private buffers (as after the host uploads
    the fields) and in the driver's order right after OCTIMF, where UKO/VKE
    share the buffers and the call copies them first."""
    from orctm_b200 import configs
    from orctm_b200.api import Instance

    over = {}
    if args.size:
        nx, ny, nz = (int(v) for v in args.size.split("x"))
        over = dict(nx=nx, ny=ny, nz=nz)
    inst = configs.make_instance("c2", index=rank, **over)
    obc = configs.make_obc(inst)
    gpu = Instance(inst, device=local)
    gpu.upload_state(configs.copy_state(inst))
    gpu.set_solver("fp64", rtol=1e-10, maxit=5000)
    gpu.set_obc(obc)
    K = max(args.steps, 1) * 10
    for s in range(args.warmup):
        gpu.obc_uv(s)
        gpu.obc_eta(s)
        gpu.step_hotpath()

    def timed(fn):
        barrier(pg)
        gpu.synchronize()
        gpu.timer_start()
        for s in range(K):
            fn(s)
        ms = gpu.timer_stop() / K
        return max_over_ranks(pg, ms)

    gpu.upload("uoo", np.asfortranarray(inst["uoo"]))   # private buffers again
    gpu.upload("voe", np.asfortranarray(inst["voe"]))
    n0 = Instance.kernel_launches()
    ms_uv = timed(gpu.obc_uv)
    launches_uv = (Instance.kernel_launches() - n0) / K
    ms_eta = timed(gpu.obc_eta)

    def uv_after_octimf(s):
        gpu.octimf()
        gpu.obc_uv(s)

    ms_uv_shared = timed(uv_after_octimf)
    for n in (0, 1):                                   # FORC_OBCS_TS records
        gpu.set_obc_ts(n, configs.make_obc_ts(inst, n))
    ms_ts = timed(lambda s: gpu.obc_ts())
    barrier(pg)
    gpu.synchronize()
    gpu.timer_start()
    for _ in range(args.steps):
        gpu.step_hotpath()
    ms_step = max_over_ranks(pg, gpu.timer_stop() / args.steps)
    cells = _band_cells(inst, obc)
    # algorithmic bytes: each band cell of UOO / VOE / ZO read and written once
    # (masks are per-column level counts, the tidal constants a few KB)
    bytes_uv = 16 * (cells["u"] + cells["v"])
    bytes_eta = 16 * cells["z"]
    bytes_ts = 2 * 16 * cells["z"] * inst["ke"]      # THO and SAO, every level
    hbm, peak_kind = peaks()
    if rank == 0:
        ach = bytes_uv / (ms_uv / 1e3) / 1e9
        line = {"metric": "open-boundary tide forcing + sponge, device time per call "
                          "(orctm_obc_uv; orctm_obc_eta beside it)",
                "value": ms_uv, "unit": "ms", "n_gpus": ws, "steps": K, "warmup": args.warmup,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": DATA,
                "config": dict(workload_config(inst), sponge_widths=obc["width"],
                               open_sides="".join(k[0].upper() for k in ("west", "east", "north",
                                                                        "south") if inst["ob"][k]),
                               ntide=obc["ntide"]),
                "obc_eta_ms": ms_eta, "obc_uv_after_octimf_ms": ms_uv_shared,
                "obc_ts_ms": ms_ts,
                "obc_ts_gbs": round(bytes_ts / (ms_ts / 1e3) / 1e9, 1),
                "step_hotpath_ms": ms_step,
                "share_of_step": (ms_uv + ms_eta + ms_ts) / ms_step,
                "band_cells": cells, "gpu_launches_per_call": launches_uv,
                "roofline": {"bound": "hbm", "kernel": "k_obc_sponge (u and v)",
                             "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                             "frac": round(ach / hbm, 4), "traffic": None,
                             "bytes_per_call": bytes_uv,
                             "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                             if peak_kind == "measured" else "fallback 6.65 TB/s"}}
        print(json.dumps(line), flush=True)
    gpu.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_e2e(gpu, inst, cells, args, ws, pg):
    """Each step: inputs copied from pinned host memory (the fields the
    hydrostatic part of the reference step produces), the hot path, the
    outputs read back (the fields the rest of the model consumes)."""
    import torch

    from orctm_b200 import configs

    st = configs.copy_state(inst)
    # the transports first (all three momentum advection routines read them),
    # then each routine's own field; the tracers last (read after the solve)
    ins = ["uko", "vke", "wo", "uoo", "voe", "wno"]
    outs = ["uoo", "voe", "wno", "pnh"]
    pinned = {}

    def pin(a):
        t = torch.empty(a.shape[::-1], dtype=torch.float64, pin_memory=True)
        v = t.numpy().T  # Fortran-ordered view
        v[...] = a
        return t, v

    for k in ins:
        pinned["in_" + k] = pin(st[k])
    for n, tr in enumerate(st["tracers"]):
        pinned[f"in_tracer{n}"] = pin(tr)
    for k in outs:
        pinned["out_" + k] = pin(np.zeros(gpu.shape(k)))
    for n in range(gpu.ntr):
        pinned[f"out_tracer{n}"] = pin(np.zeros(gpu.shape("pnh")))
    h2d = sum(pinned[k][1].nbytes for k in pinned if k.startswith("in_"))
    d2h = sum(pinned[k][1].nbytes for k in pinned if k.startswith("out_"))
    k_steps = max(2, min(args.steps, 5))

    # uploads go to the copy stream (velocities first: the momentum path
    # waits for them, the tracers land while it runs); the outputs are
    # registered so that each step downloads them as soon as they are final
    # (the momentum fields while the tracers are advected and diffused)
    outmap = {k: pinned["out_" + k][1] for k in outs}
    outmap.update({f"tracer{n}": pinned[f"out_tracer{n}"][1] for n in range(gpu.ntr)})
    gpu.set_step_outputs(outmap)

    def one():
        for k in ins:
            gpu.upload_async(k, pinned["in_" + k][1])
        for n in range(gpu.ntr):
            gpu.upload_async(f"tracer{n}", pinned[f"in_tracer{n}"][1])
        s = gpu.step_hotpath()
        gpu.wait_copies()
        return s

    one()
    barrier(pg)
    gpu.timer_start()
    for _ in range(k_steps):
        one()
    ms = gpu.timer_stop()
    ms = max_over_ranks(pg, ms)
    gpu.set_step_outputs({})
    return {"value": ws * cells * k_steps / (ms / 1e3), "unit": "cell-steps/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "steps": k_steps, "ms_per_step": ms / k_steps,
            "copies": "page-locked host buffers; uploads and downloads on a copy stream "
                      "overlapping the kernels (orctm_upload_async, orctm_set_step_outputs)"}


# ---------------------------------------------------------------- ensembles --
ENSEMBLE_OUT = ("pnh", "tracers")


def _gen_member(arg):
    """One seeded instance of config c4/c5 with the arrays a request needs
    (geometry of the descriptor, the state; shared where the state repeats a
    field).  Runs in a spawned worker process."""
    name, index = arg
    from orctm_b200 import configs

    inst = configs.make_instance(name, index=index)
    from orctm_b200.api import GEOMETRY_KEYS

    keep = ("ie", "je", "ke", "nx", "ny", "nz", "ntracers", "ob", "dt", "almzer", "aulapts",
            "aulapuv", "ah00") + GEOMETRY_KEYS
    slim = {k: inst[k] for k in keep}
    st = configs.copy_state(inst)
    del inst
    st["uko"], st["vke"], st["wo"] = st["uoo"], st["voe"], st["wno"]  # equal at the start
    return slim, st


def _members(args):
    import multiprocessing as mp

    name = "c4" if args.workload == "c4" else "c5"
    idx = [(name, k) for k in range(min(args.distinct, args.members))]
    t = time.time()
    with mp.get_context("spawn").Pool(min(len(idx), os.cpu_count() or 1)) as pool:
        pool_insts = pool.map(_gen_member, idx)
    log(f"[bench] {len(pool_insts)} distinct {name} instances generated in {time.time() - t:.1f}s")
    return [pool_insts[k % len(pool_insts)] for k in range(args.members)]


def _one_at_a_time(members, nsteps, solver):
    """The plain path: each instance created, uploaded, stepped, read back and
    destroyed before the next starts."""
    from orctm_b200.api import Instance

    lat = []
    cells = 0
    t = time.perf_counter()
    for inst, st in members:
        g = Instance(inst)
        g.upload_state(st)
        g.set_solver(solver, rtol=1e-10, maxit=5000)
        for _ in range(nsteps):
            t0 = time.perf_counter()
            g.step_hotpath()
            g.synchronize()
            lat.append((time.perf_counter() - t0) * 1e3)
        g.download("pnh")
        for n in range(g.ntr):
            g.download(f"tracer{n}")
        g.close()
        cells += (inst["ie"] - 2) * (inst["je"] - 2) * inst["ke"] * nsteps
    el = time.perf_counter() - t
    lat.sort()
    return {"value": cells / el, "elapsed_s": el, "step_ms_p50": lat[len(lat) // 2],
            "step_ms_p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]}


def run_ensemble(args, ws, rank, local, pg):
    """c4: the ensemble batch (all requests submitted together) against the
    same requests one at a time on the plain path; c5: requests arriving as a
    seeded Poisson process into the served loop.  Replicas per GPU."""
    members = _members(args)
    from orctm_b200 import serve

    nsteps = args.member_steps
    total_cells = sum((i["ie"] - 2) * (i["je"] - 2) * i["ke"] for i, _ in members) * nsteps
    res = {}
    for solver in ("fp64", "fp32_refined"):
        if args.workload == "c4":
            base = _one_at_a_time(members, nsteps, solver)
            jobs = [serve.Job(i, st, nsteps, outputs=ENSEMBLE_OUT) for i, st in members]
            barrier(pg)
            t = time.perf_counter()
            tot = serve.run_batch(jobs, device=local, slots=args.slots, solver=solver)
            el = time.perf_counter() - t
            el = max_over_ranks(pg, el)
            res[solver] = {"batched": {"value": ws * tot["cell_steps"] / el, "elapsed_s": el,
                                       "step_ms_p50": tot["step_ms_p50"],
                                       "step_ms_p99": tot["step_ms_p99"],
                                       "peak_in_flight": tot["peak_in_flight"],
                                       "failed": tot["failed"]},
                           "one_at_a_time": {**base, "value": ws * base["value"]},
                           "speedup": (tot["cell_steps"] / el) / base["value"]}
        else:
            g = np.random.Generator(np.random.PCG64(20261203 + 5))
            gaps = g.exponential(1.0 / args.rate, size=len(members))
            jobs = []
            barrier(pg)
            with serve.Server(device=local, slots=args.slots, solver=solver) as srv:
                t = time.perf_counter()
                due = 0.0
                for (inst, st), gap in zip(members, gaps):
                    due += gap
                    now = time.perf_counter() - t
                    if due > now:
                        time.sleep(due - now)
                    jobs.append(srv.submit(serve.Job(inst, st, nsteps, outputs=ENSEMBLE_OUT)))
                for j in jobs:
                    srv.wait(j)
                el = time.perf_counter() - t
                tot = srv.stats()
            q = sorted(j.stats["queued_ms"] for j in jobs)
            rl = sorted(j.stats["queued_ms"] + j.stats["run_ms"] for j in jobs)
            el = max_over_ranks(pg, el)
            res[solver] = {"value": ws * tot["cell_steps"] / el, "elapsed_s": el,
                           "step_ms_p50": tot["step_ms_p50"], "step_ms_p99": tot["step_ms_p99"],
                           "request_ms_p50": rl[len(rl) // 2],
                           "request_ms_p99": rl[min(len(rl) - 1, int(0.99 * len(rl)))],
                           "queued_ms_p50": q[len(q) // 2],
                           "queued_ms_p99": q[min(len(q) - 1, int(0.99 * len(q)))],
                           "peak_in_flight": tot["peak_in_flight"], "failed": tot["failed"]}
    if rank == 0:
        sizes = [(i["nx"], i["ny"], i["nz"]) for i, _ in members[:args.distinct]]
        head = res["fp64"]["batched"] if args.workload == "c4" else res["fp64"]
        line = {"metric": f"cell-steps/s ({args.workload} "
                          f"{'ensemble batch' if args.workload == 'c4' else 'served requests'})",
                "value": head["value"], "unit": "cell-steps/s", "n_gpus": ws,
                "steps": nsteps, "warmup": 0, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded PCG64, base seed 20261203; generators of the c1-c5 workloads)",
                "config": {"workload": f"{args.workload}: {args.members} requests over "
                                       f"{len(sizes)} distinct seeded instances, "
                                       f"{nsteps} steps each, {args.slots} slots"
                                       + (f", Poisson arrivals {args.rate}/s"
                                          if args.workload == "c5" else ""),
                           "distinct_sizes": sizes, "cell_steps_per_gpu": total_cells},
                "results": res}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
