"""Benchmark of the Gelios_2D plasma time step on B200 (cell-updates/s).

One "step" = one call of the moving-grid time step (the Go_5_komponent__MK2
form: surface tracking, rail motion, per-face HLL/exact-Godunov fluxes with
TVD reconstruction, charge-exchange source from Monte-Carlo moments,
conservative ALE update, CFL reduction) over the whole grid, inputs resident
in HBM.  Default workload: the reference's rail grid Setka(480,240,100,220,
200,200,300,300) (938,010 cells, ~1000 rays x ~1000 radial cells: the
1M-cell moving-grid configuration, whose inputs exceed the 126 MB L2), the
reference's initial field and seeded Monte-Carlo moments.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mk2_1m|mk2_200k|plain|...]

N>1 runs N independent replicas (one process per GPU, torchrun); value is
the whole-job rate, the time is the max over ranks.  --impl reference times
the reference's own CPU step (compiled from its sources, all host threads)
on the same workload and prints its line; under torchrun only rank 0 does.
For the rail-grid workloads the reference arm builds everything with the
reference itself (its constructor, TVD_prepare and Init_conditions; seeded
inputs from numpy) and loads no library of this package.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"
WORKLOADS = {
    "mk2_200k": ("moving-grid plasma step (Go_5_komponent__MK2 form) on Setka(200,100,50,100,100,100,150,150)",
                 "mk2", (200, 100, 50, 100, 100, 100, 150, 150)),
    "mk2_1m": ("moving-grid plasma step (Go_5_komponent__MK2 form) on Setka(480,240,100,220,200,200,300,300)",
               "mk2", (480, 240, 100, 220, 200, 200, 300, 300)),
    "mk2_8k": ("moving-grid plasma step (Go_5_komponent__MK2 form) on Setka(30,7,11,20,60,20,40,40)",
               "mk2", (30, 7, 11, 20, 60, 20, 40, 40)),
    "plain": ("plain single-fluid step (Go_stationary form), polar 180x120, r=1..600", "plain", None),
    "k5_200k": ("plasma + four hydrogen fluids (Go_5_komponent form) on Setka(200,100,50,100,100,100,150,150)",
                "k5", (200, 100, 50, 100, 100, 100, 150, 150)),
    "inner_200k": ("inner fixed-grid region step (Go_stationary_5_komponent_inner_MK2 form): All_Cells_Inner "
                   "(centroid radius <= R111) of Setka(200,100,50,100,100,100,150,150)", "inner",
                   (200, 100, 50, 100, 100, 100, 150, 150)),
    "mhd_200k": ("ion MHD fluid (HLLD) + pickup protons (HLLC) on the moving grid Setka(200,100,50,100,100,100,"
                 "150,150): LISM B=0.01 at 30 deg, seeded fixed charge-exchange sources", "mhd",
                 (200, 100, 50, 100, 100, 100, 150, 150)),
    "mhd_8k": ("ion MHD fluid (HLLD) + pickup protons (HLLC) on the moving grid Setka(30,7,11,20,60,20,40,40): "
               "LISM B=0.01 at 30 deg, seeded fixed charge-exchange sources", "mhd", (30, 7, 11, 20, 60, 20, 40, 40)),
    "mhd_1m": ("ion MHD fluid (HLLD) + pickup protons (HLLC) on the moving grid Setka(480,240,100,220,200,200,300,"
               "300): LISM B=0.01 at 30 deg, seeded fixed charge-exchange sources", "mhd",
               (480, 240, 100, 220, 200, 200, 300, 300)),
    "sweep64": ("64 independent MHD + pickup-proton instances (FP32 fluxes, FP64 accumulation), Setka(200,100,50,100,"
                "100,100,150,150) scaled by U(0.5,1.4) per instance (~50k..~400k cells, ~11M in all), seeded inflow "
                "u~U(0.04,0.08), rho~U(0.002,0.01), Mach~U(1.5,3), |B|~U(0,0.02), angle~U(0,60 deg)", "sweep", None),
    "sweep16": ("16 independent moving-grid instances, Setka(200,100,50,100,100,100,150,150) scaled by "
                "U(0.5,1.4) per instance (~50k..~400k cells each), batched on each GPU", "sweep", None),
}
# Algorithmic bytes per cell update (each datum moved once per step):
#   MK2 form: 8*(2*5) state + 8*19 Monte-Carlo moments + 16*(1+1) points (x,y,x2,y2)
#             + 8 written point coordinate + 4*4 neighbour indices = 288 B
#   plain form: 8*(2*5) + 16 points + 4*4 indices = 112 B
#   four-fluid form: 8*(2*21) state (plasma 5 + hydrogen 16) + 16*(1+1) points
#             + 8 written point coordinate + 4*4 neighbour indices = 392 B
#   MHD + pickup form: 8*(2*13) state (ions ro, p, u, v, w, Bx, By, Bz, Q; pickup
#             ro, p, u, v) + 8*3 fixed sources + 16*(1+1) points + 8 written point
#             coordinate + 4*4 neighbour indices = 288 B
#   inner form: 8*(2*5) state + 8*19 Monte-Carlo moments + 16 points (fixed
#             grid) + 4*4 neighbour indices = 264 B
BYTES_PER_CELL = {"mk2": 288, "plain": 112, "k5": 392, "mhd": 288, "inner": 264}
STEP_KERNELS = {
    "mk2": "whole moving-grid step, pipelined: source, tracked flux, face units (reconstruction + flux, "
           "autotuned arrangement), update of the cells the next motion reads, then the next step's dt, "
           "surface_faces, rails, tracked recon + solve beside the update of the other cells "
           "(CUDA graphs, 4 streams; one commit per call)",
    "plain": "whole plain step: stationary_persistent_kernel (face units, cell update, dt; all steps of a call "
             "in one cooperative launch)",
    "k5": "whole four-fluid step: centroid, surface_faces, rails, k5_cell, commit",
    "mhd": "whole MHD + pickup step: surface_faces, rails, mhd_face, mhd_update, commit",
    "inner": "whole inner-region step: inner_cell + dt_finalize",
}


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def workload_config(name: str, cells: int, counted: int, faces: int, points: int, world: int) -> dict:
    desc, form, _ = WORKLOADS[name]
    return {"workload": desc, "cells": int(cells), "cells_updated_per_step": int(counted), "faces": int(faces),
            "points": int(points),
            "l2": ("inputs larger than L2 (126 MB), not flushed" if name.endswith("_1m") else
                   "flushed (256 MiB write) before each timed call of 100 steps; the few-MB state stays "
                   "L2-resident within a call" if form in ("plain", "inner") else
                   "flushed between timed steps (256 MiB write)"),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def build_workload(name: str):
    import gelios_2d_b200 as g
    from gelios_2d_b200 import _native as N
    from gelios_2d_b200 import workloads as W

    desc, form, dims = WORKLOADS[name]
    if form == "mk2":
        mesh = g.Mesh.setka(*dims)
        params = N.reference_params()
        st0 = W.init_conditions_reference(mesh)
        mc = W.mc_fields(mesh, seed=9)
        counted = W.counted_cells_mk2(mesh, params)
    elif form == "inner":
        mesh = g.Mesh.setka(*dims)
        params = N.reference_params()
        st0 = W.init_conditions_reference(mesh)
        mc = W.mc_fields(mesh, seed=9)
        inner = mesh.inner_cells(params.R111)
        counted = int(np.count_nonzero(mesh["cell_type"][inner] != 5))  # C_centr cells are copied
    elif form == "mhd":
        # `mc` carries (boundary data, extra rows (8, n_cells), fixed sources)
        mesh = g.Mesh.setka(*dims)
        params = N.reference_params()
        st0 = W.init_conditions_reference(mesh)
        mp = W.mhd_params()
        mc = (mp, W.mhd_initial(mesh, st0, mp), W.mhd_sources(mesh, seed=17))
        counted = W.counted_cells_mk2(mesh, params)
    elif form == "k5":
        # `mc` carries the hydrogen fluids (16, n_cells) for this form
        mesh = g.Mesh.setka(*dims)
        params = N.reference_params()
        st0 = W.init_conditions_reference(mesh)
        mc = W.hydrogen_fields(mesh, seed=3)
        counted = W.counted_cells_mk2(mesh, params)
    else:
        mesh = W.plain_mesh()
        params = W.plain_params()
        st0 = W.plain_initial(mesh, params, seed=2024)
        mc = None
        counted = W.counted_cells_stationary(mesh)
    return desc, form, dims, mesh, params, st0, mc, counted


class ClockSampler:
    """nvidia-smi samples of SM clock / power / throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


PROFILE_SUMMARY = {"mk2_200k": "mk2_step_setka200k.md", "mk2_1m": "mk2_step_setka1m.md",
                   "plain": "stationary_step_polar180x120.md", "mhd_200k": "mhd_step_setka200k.md",
                   "mhd_1m": "mhd_step_setka1m.md"}


def ncu_traffic(workload: str):
    """DRAM bytes (read + write) of all kernels of one step, from the
    committed ncu summary of this workload (line `dram_bytes_per_step: N`)."""
    name = PROFILE_SUMMARY.get(workload)
    p = ROOT / "profiles" / name if name else None
    if not p or not p.exists():
        return None
    import re

    m = re.search(r"^dram_bytes_per_step:\s*([0-9.eE+]+)", p.read_text(), re.M)
    return float(m.group(1)) if m else None


def cpu_oracle_mhd_rate(mesh, params, st0, mc, counted, budget_s=12.0, max_steps=200):
    """The MHD + pickup form has no reference step: its CPU baseline is the
    oracle's restatement (go_mhd, one thread) on the same grid and inputs."""
    from oracle import oracle as O

    go = O.GoParams(**{n: getattr(params, n) for n, _ in O.GoParams._fields_ if n != "pad_"}, pad_=0)
    ora = O.Oracle(go, mesh)
    for b in (0, 1):
        ora.set_state(b, st0)
        ora.set_mhd(b, mc[1])
    ora.set_sources(*mc[2])
    mp = mc[0].as_dict()
    t0 = time.perf_counter()
    ora.mhd(mp, 1)
    one = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    ora.mhd(mp, steps)
    el = time.perf_counter() - t0
    return counted * steps / el, steps, 1, el


RAIL_FORMS = ("mk2", "inner", "k5")


def reference_workload(name: str):
    """The rail-grid workload `name` built by the reference alone (its own
    constructor, TVD_prepare and Init_conditions in oracle/_ref; seeded
    inputs from numpy): nothing of this package is imported or loaded."""
    from oracle import ref_workload as RW

    _, form, dims = WORKLOADS[name]
    return RW.build(dims, form)


def cpu_reference_rate(mesh, params, st0, mc, counted, form, budget_s=12.0, max_steps=200, threads=None,
                       rw=None):
    """The reference's own step (compiled from its sources, all host threads)
    on the same workload: cell-updates/s over a bounded number of steps.
    Rail-grid forms run on `rw` (a reference_workload); the plain form on
    reference objects made from `mesh`; the MHD form, which has no
    reference step, on the oracle's restatement."""
    if form == "mhd":
        return cpu_oracle_mhd_rate(mesh, params, st0, mc, counted, budget_s, max_steps)
    from oracle import ref

    threads = threads or os.cpu_count() or 1
    ref.set_threads(threads, fast=True)
    if form in RAIL_FORMS:
        if rw is None:
            raise ValueError("rail-grid forms run on a reference_workload")
        S, counted = rw.S, rw.counted
    else:
        S = ref.RefSetka.from_mesh(mesh, fast=True)
        S.tvd_prepare()
        S.set_state(0, st0)
        S.set_state(1, st0)
    run = {"mk2": S.go_mk2, "k5": S.go_5_komponent, "inner": S.go_inner_mk2}.get(form, S.go_stationary)
    # keep the reference's printf diagnostics off our stdout
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        t0 = time.perf_counter()
        run(1)
        one = time.perf_counter() - t0
        steps = int(max(1, min(max_steps, budget_s / max(one, 1e-6))))
        t0 = time.perf_counter()
        run(steps)
        el = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)
    return counted * steps / el, steps, threads, el


def load_inputs(S, form, st0, mc):
    """par[0] = par[1] = st0, plus the form's extra inputs: Monte-Carlo
    moments (moving grid) or the hydrogen fluids (four-fluid form)."""
    S.set_par(0, st0)
    S.set_par(1, st0)
    if form == "k5":
        S.set_hydrogen(0, mc)
        S.set_hydrogen(1, mc)
    elif form == "inner":
        S.set_mc(*mc)
        S.build_inner_list()
    elif form == "mhd":
        S.set_mhd_params(mc[0])
        S.set_mhd(0, mc[1])
        S.set_mhd(1, mc[1])
        S.set_sources(*mc[2])
    elif mc is not None:
        S.set_mc(*mc)


def fp32_flux_errors(mesh, params32, st0, mc, fcode, device, counts=(1, 100, 2000), form="") -> dict:
    """L1 and Linf relative errors of rho, p, u, v of the FP32-flux form
    against the FP64 path (itself within 1e-12 per step of the reference's
    CPU step) after 1, 100 and 2000 steps from the same initial state."""
    import numpy as np

    import gelios_2d_b200 as g
    from gelios_2d_b200 import _native as N

    params64 = params32.copy(precision=N.PREC_FP64)
    out = {"against": "FP64 device path"}
    for n in counts:
        res = []
        for prm in (params32, params64):
            S = g.Setka(mesh, prm, device=device)
            load_inputs(S, form, st0, mc)
            st = S.step(fcode, n)
            r = S.par(st.result_buf)
            if form == "mhd":
                r = np.concatenate([r, S.mhd(st.result_buf)])
            res.append(r)
            S.close()
        a, b = res
        errs = {}
        names = ("rho", "p", "u", "v") if form != "mhd" else ("rho", "p", "u", "v", None, "w", "Bx", "By", "Bz")
        for k, name in enumerate(names):
            if name is None:
                continue
            d = np.abs(a[k] - b[k])
            errs[name] = {"L1": float(d.sum() / max(np.abs(b[k]).sum(), 1e-300)),
                          "Linf": float(d.max() / max(np.abs(b[k]).max(), 1e-300))}
        if form == "mhd":
            # vector scales: w (zero at the start) against the ion speed, each
            # field component against |B|
            spd = np.sqrt(b[2] ** 2 + b[3] ** 2 + b[5] ** 2)
            bm = np.sqrt(b[6] ** 2 + b[7] ** 2 + b[8] ** 2)
            dw = np.abs(a[5] - b[5])
            errs["w/|u|"] = {"L1": float(dw.sum() / max(spd.sum(), 1e-300)),
                             "Linf": float(dw.max() / max(spd.max(), 1e-300))}
            db = np.sqrt((a[6] - b[6]) ** 2 + (a[7] - b[7]) ** 2 + (a[8] - b[8]) ** 2)
            errs["B/|B|"] = {"L1": float(db.sum() / max(bm.sum(), 1e-300)),
                             "Linf": float(db.max() / max(bm.max(), 1e-300))}
        out[str(n)] = errs
    return out


def time_to_residual(workload, mesh, params, st0, mc, form, fcode, device, tol, counted, max_steps=5_000_000,
                     check_every=10_000) -> dict:
    """Wall time from the seeded (cold) initial field until the density's L1
    residual per unit time, sum|ro(n+1) - ro(n)| / (dt sum|ro(n+1)|), is at
    most tol (checked every check_every steps), and the reference CPU step's
    time for the same number of steps, projected from a bounded sample."""
    import gelios_2d_b200 as g

    S = g.Setka(mesh, params, device=device)
    load_inputs(S, form, st0, mc)
    S.synchronize()
    t0 = time.perf_counter()
    steps, r, dt = S.run_to_residual(fcode, tol, max_steps, check_every)
    gpu_s = time.perf_counter() - t0
    S.close()
    out = {"tol": tol, "definition": "sum|ro(n+1)-ro(n)| / (dt * sum|ro(n+1)|), checked every "
                                      f"{check_every} steps", "start": "cold (the workload's seeded initial field)",
           "reached": r <= tol, "steps": steps, "residual": r, "dt": dt, "gpu_s": gpu_s}
    try:
        rw = reference_workload(workload) if form in RAIL_FORMS else None
        rate, n, threads, el = cpu_reference_rate(mesh, params, st0, mc, counted, form, budget_s=10.0, rw=rw)
        out["reference_cpu_s_projected"] = steps * counted / rate
        out["reference_cpu_sample"] = f"{n} steps on {threads} host threads ({el:.1f} s)"
    except Exception as e:  # the reference library must be prebuilt
        out["reference_cpu_s_projected"] = None
        out["reference_cpu_sample"] = f"unavailable: {e}"
    return out


def march_record(mesh, params, st0, mc, fcode, device, total, every, form="mk2") -> list:
    """A moving-grid step (the MK2 form, or the MHD + pickup form) marched
    from the workload's initial field in calls of `every` steps (each call
    restarts dt at dt0, as the reference's time loop does), recording after
    each call: the step residual per unit time (sum|ro(n+1)-ro(n)| / (dt
    sum|ro(n+1)|), which contains the volume change of moving cells), the
    operator residual with the grid held still (gelios_operator_residual:
    (ion) mass flux balance per unit volume, face speeds 0), the largest and
    the mean point displacement per step over the call, dt and the status
    flags."""
    import gelios_2d_b200 as g

    S = g.Setka(mesh, params, device=device)
    load_inputs(S, form, st0, mc)
    x0, y0 = S.points()
    out = []
    done = 0
    while done < total:
        n = min(every, total - done)
        st = S.step(fcode, n)
        done += n
        x1, y1 = S.points()
        mv = np.hypot(x1 - x0, y1 - y0)
        x0, y0 = x1, y1
        rb = int(st.result_buf)
        r_step = S.residual(rb) / st.dt if st.dt > 0 else float("nan")
        rec = {"steps": done, "dt": float(st.dt), "flags": int(st.flags), "step_residual_per_time": float(r_step),
               "operator_residual_per_time": float(S.operator_residual(rb, fcode)),
               "point_move_per_step_max": float(np.max(mv) / n), "point_move_per_step_mean": float(np.mean(mv) / n)}
        out.append(rec)
        if st.flags or not np.isfinite(r_step):
            break
    S.close()
    return out


def run_sweep(args, rank: int, world: int, local: int) -> None:
    """The sweep workload: instances partitioned over the ranks by cell count,
    each rank steps its instances together (one context and graph per
    instance); value = all cells updated / the slowest rank's device time."""
    import torch

    import gelios_2d_b200 as g  # noqa: F401
    from gelios_2d_b200 import sweep as sw
    from gelios_2d_b200 import workloads as W
    from gelios_2d_b200.replicas import max_over_ranks, whole_job_rate

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = dist_mod
    torch.cuda.set_device(local)
    from gelios_2d_b200 import _native as N

    mhd = args.workload == "sweep64"
    n_inst, seed = (64, 43) if mhd else (16, 41)
    seeds = W.splitmix64(seed, n_inst)
    sizes = []  # estimated cells per instance, to partition before building
    for i in range(n_inst):
        f = 0.5 + 0.9 * float(seeds[i])
        sizes.append(f * f)
    mine = sw.partition(sizes, world)[rank]
    if mhd:
        inst = sw.instance_set_mhd(n_inst, seed=seed, scale=(0.5, 1.4), only=mine)
        inst = [(m, p.copy(precision=N.PREC_FP32_FLUX), s, x) for m, p, s, x in inst]
    else:
        inst = sw.instance_set(n_inst, seed=seed, scale=(0.5, 1.4), only=mine)
    counted = sum(W.counted_cells_mk2(m, p) for m, p, _, _ in inst)
    cells = sum(m.n_cells for m, _, _, _ in inst)
    batched = mhd and args.sweep_mode in ("batched", "persistent")
    call_steps = max(1, int(args.sweep_call_steps))
    B = sw.Sweep(inst, device=local, form=N.FORM_MHD_PUI if mhd else N.FORM_MK2)
    tuned = None
    if mhd and not batched:  # per-instance launch shape and enqueue order (the sweep's autotuner)
        res = B.autotune(reps=3)
        tuned = {}
        for v, _ in res:
            tuned[str(v)] = tuned.get(str(v), 0) + 1
    schedule = None
    if batched:  # one launch per phase over the instances of a group (gelios_batch)
        B.enable_batch(args.sweep_groups)
        if args.sweep_mode == "persistent":
            # the batch's autotuner: per-phase graph or one persistent kernel at
            # each co-resident block count (its trial steps advance the instances)
            schedule = B.autotune_batch(2)
    streams = [torch.cuda.ExternalStream(S.stream_handle(), device=local) for S in B.items]
    s0 = torch.cuda.current_stream(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def one(ev=None):
        flush.fill_(1.0)
        start = torch.cuda.Event(enable_timing=True)
        start.record(s0)
        for st in streams:
            st.wait_event(start)
        B.step_async(call_steps)
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            s0.wait_event(e)
        end = torch.cuda.Event(enable_timing=True)
        end.record(s0)
        if ev is not None:
            ev.append((start, end))
        if batched:  # every context of a group reports the group's launches
            return sum(B.items[p[0]].launches() for p in B._groups)
        return sum(S.launches() for S in B.items)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize(local)
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    evs, launches = [], 0
    for _ in range(args.steps):
        launches += one(evs)
    torch.cuda.synchronize(local)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dist, f"cuda:{local}")
    counted_all = counted
    if dist:
        t = torch.tensor([float(counted)], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t)
        counted_all = float(t.item())
    value = counted_all * args.steps * call_steps / (total_ms / 1000.0)
    peak, peak_kind = measured_peaks()
    bpc = BYTES_PER_CELL["mhd" if mhd else "mk2"]
    achieved = bpc * counted_all / world / (total_ms / args.steps / call_steps / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps / call_steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64 (fp32 flux)" if mhd else "f64",
        "data": "synthetic (seeded instances: grid scale, inflow, initial field, " +
                ("LISM field, charge-exchange sources)" if mhd else "Monte-Carlo moments)"),
        "config": {"workload": WORKLOADS[args.workload][0], "instances": n_inst, "instances_on_rank0": len(inst),
                   "cells_rank0": int(cells), "cells_updated_per_step": int(counted_all),
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"instances partitioned over {world} GPU(s)",
                   "autotune_variants_rank0": tuned, "steps_per_call": call_steps,
                   "batch_schedule_rank0": schedule,
                   "mode": ("persistent: autotuned per group between one launch per phase (schedule 0) and one "
                            "cooperative kernel over all steps of a call (schedule k: k blocks per SM)")
                           if args.sweep_mode == "persistent" and mhd else
                           "batched: one launch per phase over all instances, one CUDA graph per step" if batched
                           else "one context and captured step graph per instance, enqueued together"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "batched moving-grid steps of all instances on a GPU",
                     "bytes_per_cell": bpc, "avg_launch_us": total_ms / args.steps / call_steps * 1000.0,
                     "peak_kind": f"{peak_kind} hbm_gbs (burst copy)"},
        "clocks": clocks,
    }
    B.close()
    if mhd and rank == 0 and args.sweep_errors > 0:
        # FP32-flux errors of the sweep's own instances against their FP64 steps
        per = []
        for mesh, p32, st0, extra in inst[: args.sweep_errors]:
            e = fp32_flux_errors(mesh, p32, st0, extra, N.FORM_MHD_PUI, local, form="mhd")
            e["cells"] = int(mesh.n_cells)
            per.append(e)
        worst = {}
        for e in per:
            for n, errs in e.items():
                if not isinstance(errs, dict):
                    continue
                w = worst.setdefault(n, {})
                for name, v in errs.items():
                    o = w.setdefault(name, {"L1": 0.0, "Linf": 0.0})
                    o["L1"] = max(o["L1"], v["L1"])
                    o["Linf"] = max(o["Linf"], v["Linf"])
        line["fp32_flux_errors"] = {"against": "FP64 device path, same instance and initial state",
                                    "instances": len(per), "worst_over_instances": worst, "per_instance": per}
    if mhd and rank == 0 and args.sweep_march:
        # config-4 instances (FP32 fluxes) marched from their cold start: step
        # and operator residuals per call of --march-every steps; the
        # smallest, the median and the largest instance of this rank
        order = sorted(range(len(inst)), key=lambda i: inst[i][0].n_cells)
        pick = sorted({order[0], order[len(order) // 2], order[-1]})
        line["march"] = []
        for i in pick:
            mesh, p32, st0, extra = inst[i]
            rec = march_record(mesh, p32, st0, extra, N.FORM_MHD_PUI, local, args.sweep_march, args.march_every, "mhd")
            line["march"].append({"instance_on_rank0": i, "cells": int(mesh.n_cells), "record": rec})
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_warm_start(args, rank: int) -> None:
    """The learned warm start on the plain problem (the Go_stationary form on
    the polar grid of --ws-grid): converged training states from the batched
    solver, the network trained on the GPU, then held-out parameter sets
    marched to an L1 residual per unit time of --ws-tol from the cold start,
    the nearest training state, the network's prediction and the nearest
    state moved by the network.  value = wall time of the batched warm
    (network) FP64 solve of all held-out instances."""
    if rank != 0:
        return
    from gelios_2d_b200 import _native as N
    from gelios_2d_b200 import warmstart as W
    from gelios_2d_b200.mesh import Mesh

    nt, nr = (int(v) for v in args.ws_grid.split("x"))
    mesh = Mesh.polar(nt, nr, 1.0, 600.0)
    t0 = time.perf_counter()
    out, _ = W.experiment(mesh, n_train=args.ws_train, n_test=args.ws_test, tol=args.ws_tol,
                          train=dict(iters=args.ws_iters), n_serial=2, fp32_max_steps=100_000)
    total = time.perf_counter() - t0
    theta = [0.005, 0.06, 2.0, 1.0, 10.0]
    params = W.inflow_params(theta)
    st0 = W.cold_state(mesh, params)
    counted = int(np.sum(mesh["cell_type"] != 5))
    cpu = None
    if not args.no_cpu_baseline:
        try:
            rate, steps, threads, el = cpu_reference_rate(mesh, params, st0, None, counted, "plain", budget_s=10.0)
            proj = out["cold_fp64"]["steps_mean"] * counted * args.ws_test / rate
            cpu = {"value": proj, "unit": "s", "cores": threads, "kind": "reference",
                   "sample": f"{steps} reference Go_stationary steps on {threads} host threads ({el:.1f} s); "
                             f"projected for cold solves of the {args.ws_test} held-out instances one after another"}
        except Exception as e:  # the reference library must be prebuilt
            cpu = {"value": None, "unavailable": str(e)}
    warm = out["warm_fp64"]
    line = {"metric": f"wall time to L1 residual {args.ws_tol:g} per unit time, {args.ws_test} held-out instances "
                      "(batched, network warm start)",
            "value": warm["wall_s"], "unit": "s", "n_gpus": 1, "steps": int(sum(warm["steps"])), "warmup": 0,
            "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 step; bf16 GEMMs with fp32 accumulation in the network",
            "data": "synthetic (seeded inflow parameter sets, seeded initial fields)",
            "config": {"workload": f"learned warm start, plain problem on the {nt} x {nr} polar grid",
                       "cells": int(mesh.n_cells), "n_train": args.ws_train, "n_test": args.ws_test,
                       "tol": args.ws_tol, "network": "7 inputs + 24 Fourier features -> 5 x 256 GELU -> 5",
                       "l2": "state and network resident in L2 (small instances)"},
            "warm_start": out, "wall_s_total": total, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mk2_1m", choices=sorted(WORKLOADS) + ["warm_start"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32flux"])
    # moving-grid / MHD forms: use this variant of the face units + update instead of autotuning
    # (the autotuner times kernels alone; under a profiler its choice would differ from the plain run's)
    ap.add_argument("--variant", type=int, default=None)
    # sweep64 only: one context and captured step graph per instance, autotuned and enqueued together
    # (default), or gelios_batch: one launch per phase over the instances of each of --sweep-groups groups
    ap.add_argument("--sweep-mode", default="contexts", choices=["contexts", "batched", "persistent"])
    ap.add_argument("--sweep-groups", type=int, default=1)
    ap.add_argument("--sweep-call-steps", type=int, default=1, help="steps per timed call of the sweep")
    ap.add_argument("--sweep-march", type=int, default=0,
                    help="sweep64: march three instances this many steps, recording their residuals")
    ap.add_argument("--sweep-errors", type=int, default=0,
                    help="sweep64: FP32-flux L1/Linf errors of this many instances after 1, 100, 2000 steps")
    # wall time to an L1 residual per unit time (cold start), reported beside the rate
    ap.add_argument("--residual", type=float, default=None)
    # moving-grid workloads: march this many steps from the initial field, recording the step residual, the
    # operator residual (grid held still) and the point motion after every call of --march-every steps
    ap.add_argument("--march", type=int, default=None)
    ap.add_argument("--march-every", type=int, default=10000)
    # warm_start only: polar grid, training / held-out parameter sets, residual tolerance, training steps
    ap.add_argument("--ws-grid", default="90x60")
    ap.add_argument("--ws-train", type=int, default=256)
    ap.add_argument("--ws-test", type=int, default=32)
    ap.add_argument("--ws-tol", type=float, default=1e-6)
    ap.add_argument("--ws-iters", type=int, default=16000)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 only
    if args.workload == "warm_start":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no warm start; its cold "
                              "solves are projected in this workload's cpu_baseline"}))
            return
        run_warm_start(args, rank)
        return
    if args.workload in ("sweep16", "sweep64"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the sweep workload has no reference arm; "
                              "its instances are the moving-grid step timed by the default workload"}))
            return
        run_sweep(args, rank, world, local)
        return
    _, form, _ = WORKLOADS[args.workload]
    cpu_kind = "port" if form == "mhd" else "reference"
    cpu_what = "the oracle's restatement (no reference step exists)" if form == "mhd" else "the reference step"
    if args.impl == "reference":
        if form in RAIL_FORMS:  # built and stepped by the reference alone
            rw = reference_workload(args.workload)
            config = workload_config(args.workload, rw.n_cells, rw.counted, rw.n_faces, rw.n_points, world)
            rate, steps, threads, el = cpu_reference_rate(None, None, None, None, rw.counted, form, rw=rw)
        else:
            desc, form, dims, mesh, params, st0, mc, counted = build_workload(args.workload)
            config = workload_config(args.workload, mesh.n_cells, counted, mesh.n_faces, mesh.n_points, world)
            rate, steps, threads, el = cpu_reference_rate(mesh, params, st0, mc, counted, form)
        line = {"metric": METRIC, "value": rate, "unit": "cell-updates/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * el / steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": config,
                "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": cpu_kind,
                                 "sample": f"{steps} steps of {cpu_what} on the full grid ({el:.1f} s)"},
                "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    desc, form, dims, mesh, params, st0, mc, counted = build_workload(args.workload)
    config = workload_config(args.workload, mesh.n_cells, counted, mesh.n_faces, mesh.n_points, world)

    import torch

    import gelios_2d_b200 as g
    from gelios_2d_b200 import _native as N
    from gelios_2d_b200.replicas import max_over_ranks, whole_job_rate

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = dist_mod
    device = local
    torch.cuda.set_device(device)
    if args.precision == "fp32flux":
        params = params.copy(precision=N.PREC_FP32_FLUX)
    S = g.Setka(mesh, params, device=device)
    load_inputs(S, form, st0, mc)
    tuned = None
    fcode = {"mk2": N.FORM_MK2, "k5": N.FORM_5_KOMPONENT, "mhd": N.FORM_MHD_PUI,
             "inner": N.FORM_INNER_MK2}.get(form, N.FORM_STATIONARY)
    if form in ("mhd", "mk2") and args.variant is not None:  # a fixed arrangement (profiling runs)
        S.set_variant(fcode, args.variant)
        tuned = {"variant": args.variant, "fixed": True}
    elif form in ("mhd", "mk2"):  # launch shape of the face kernel picked on this grid (the library's autotuner)
        v, tms = S.autotune(fcode, reps=3)
        tuned = {"variant": v, "face_kernel_ms": tms}
    stream = torch.cuda.ExternalStream(S.stream_handle(), device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
    do_flush = not args.workload.endswith("_1m")
    # steps per timed call: 10 on the 1M-cell grids (inputs larger than L2);
    # 100 on the plain grid, whose 2.4 MB state stays L2-resident within a
    # call as in the reference's long step loops (L2 flushed before each
    # call; the call runs all its steps in one cooperative launch); 1 else
    steps_per_call = 10 if not do_flush else (100 if form in ("plain", "inner") else 1)

    def one(timed_events=None):
        if do_flush:
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
        if timed_events is not None:
            timed_events[0].record(stream)
        S.step_async(fcode, steps_per_call)
        if timed_events is not None:
            timed_events[1].record(stream)
        return S.launches()

    for _ in range(args.warmup):
        one()
    S.synchronize()

    sampler = ClockSampler(device)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    sampler.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    for k in range(args.steps):
        launches += one(evs[k])
    S.synchronize()
    torch.cuda.synchronize(device)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dist, f"cuda:{device}")
    n_steps_total = args.steps * steps_per_call
    value = whole_job_rate(counted * n_steps_total, world, total_ms / 1000.0)

    # per-phase device times, from a separate untimed pass with events
    # between the phases (the timed pass replays the captured step)
    S.set_phase_timing(True)
    S.phase_times(reset=True)
    for _ in range(min(args.steps, 20)):
        one()
    S.synchronize()
    phases = S.phase_times(reset=True)
    S.set_phase_timing(False)

    # end to end through the public API: every step takes its input state
    # from pinned host memory and leaves its result there
    # (gelios_run_streamed: the copies of the next input and of the previous
    # result overlap the step; the bytes moved per step are the full state)
    block = st0 if form not in ("k5", "mhd") else np.concatenate([st0, mc if form == "k5" else mc[1]])
    block = np.ascontiguousarray(block, dtype=np.float64)
    ring = 4
    ins = [torch.from_numpy(block.copy()).pin_memory().numpy() for _ in range(ring)]
    outs = [torch.empty(block.shape, dtype=torch.float64).pin_memory().numpy() for _ in range(ring)]
    e2e_bytes = int(block.nbytes)
    e2e_steps = max(3, min(args.steps, 50))
    host_in = [ins[k % ring] for k in range(e2e_steps)]
    host_out = [outs[k % ring] for k in range(e2e_steps)]
    S.run_streamed(fcode, host_in[:2], host_out[:2])  # staging buffers and step graphs
    S.synchronize()
    t0 = time.perf_counter()
    S.run_streamed(fcode, host_in, host_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{device}")
    e2e_value = whole_job_rate(counted * e2e_steps, world, e2e_s)

    # roofline of the step as a whole: its kernels run concurrently on two
    # streams (one CUDA graph per step), so the unit of work the algorithmic
    # bytes are counted for is the step
    step_s = total_ms / n_steps_total / 1000.0
    bpc = BYTES_PER_CELL[form]
    achieved = bpc * counted / step_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(args.workload)
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / n_steps_total, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64 (fp32 flux)",
        "data": "synthetic (seeded initial field and Monte-Carlo moments)", "config": config,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": e2e_bytes,
                "d2h_bytes_per_step": e2e_bytes,
                "moved_per_step": "the step's full state rows in from pinned host memory and out again "
                                  f"({block.shape[0]} rows x {block.shape[1]} cells, gelios_run_streamed)" +
                                  ("; the Monte-Carlo moments (19 doubles per cell) stay resident: the coupled "
                                   "host code refreshes them once per global iteration, not per step"
                                   if form in ("mk2", "inner") else "")},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": STEP_KERNELS[form], "bytes_per_cell": bpc,
                     "avg_launch_us": step_s * 1e6, "peak_kind": f"{peak_kind} hbm_gbs (burst copy)"},
        "phases_ms": {k: v[0] for k, v in phases.items()},
        "autotune": tuned,
        "clocks": clocks,
    }
    if args.precision == "fp32flux" and rank == 0:
        line["fp32_flux_errors"] = fp32_flux_errors(mesh, params, st0, mc, fcode, device, form=form)
    if args.march is not None and rank == 0 and form in ("mk2", "mhd"):
        line["march"] = march_record(mesh, params, st0, mc, fcode, device, args.march, args.march_every, form)
    if args.residual is not None and rank == 0:
        line["time_to_residual"] = time_to_residual(args.workload, mesh, params, st0, mc, form, fcode, device,
                                                    args.residual, counted)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rw = reference_workload(args.workload) if form in RAIL_FORMS else None
            rate, steps, threads, el = cpu_reference_rate(mesh, params, st0, mc, counted, form, rw=rw)
            line["cpu_baseline"] = {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": cpu_kind,
                                    "sample": f"{steps} steps of {cpu_what} on the full grid ({el:.1f} s)"}
        except Exception as e:  # the reference library must be prebuilt
            line["cpu_baseline"] = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
