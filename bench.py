#!/usr/bin/env python3
"""Benchmark of the level-set toolbox hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): 256^3 interior cells on [-1,1]^3 (3 ghost cells), union
of 6 seeded spheres, normal-velocity motion F = 1 + 0.2 sin(4 pi x) sin(4 pi y)
sin(4 pi z), HJ-WENO5 + Godunov + TVD-RK3 at CFL 0.5 with the CFL dt of every
step, reinitialization (20 TVD-RK3 pseudo-steps, dt = 0.5 dx) after every 10th
step.  One benchmark step = one physical time step (CFL dt + 3 stages), the
reinitialization cost included at its cadence.  Metric: cell-updates/s (one
interior cell advanced one full step), FP64.

Our arm prints one JSON line with value (device-resident fused drivers, FP64
fast arithmetic), the FP32 form beside it (with its error against the FP64
run), e2e (the same steps through the C ABI with the level set and speed on
pinned host memory, copied in and out every step), the roofline of the
dominant kernel, the CFL-dt kernel count and the reference's CPU toolbox timed
on this host.  Beside it: the batched, adjoint, deformation and per-routine
toolbox legs, and the fast marching leg (distance function, extension
fields and Eikonal solver with the reference's march values, 128^3 and 256^3,
against the CPU oracle of the reference's heap march).  Under torchrun every rank runs a replica on its own GPU
(weak scaling, no data-path collective).

``--impl reference`` times the reference's own toolbox routines (translated
from its Fortran sources, oracle/_ref) on all host cores, patch-decomposed as
the reference's parallel package does, on the same full workload (a bounded
number of timed steps); rank 0 alone runs it.
"""
import argparse
import ctypes
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

METRIC = ("cell-updates/s, plain FP64 vs FP32/batched at ≤1e-5 err; "
          "% HBM; adjoint/fwd")
UNIT = "cell-updates/s"
N_CELLS = 256
WORKLOAD = ("256^3 normal-velocity level set (6 spheres, F = 1 + 0.2 sin sin sin), "
            "HJ-WENO5 + Godunov + TVD-RK3, CFL 0.5, reinit every 10 steps x 20")



# DRAM bytes (read + write) per launch and FP64-pipe utilisation of the fused
# stage kernels on the 256^3 workload, from the ncu capture summarised in
# profiles/k_stage_pairs_config2_256.md (distinct phi_s and phi^n)
NCU_TRAFFIC = {"stage_reinit_rk32": 394.9e6, "stage_normal_rk32": 541.5e6}
NCU_FP64_PIPE = {"stage_reinit_rk32": 62.5, "stage_normal_rk32": 63.5}
# FP64 thread instructions per cell of the same kernels (ncu op counters
# smsp__sass_thread_inst_executed_op_fp64_pred_on, the same capture's
# profile command) and the B200's FP64 lanes per SM
NCU_FP64_OPS_PER_CELL = {"stage_reinit_rk32": 266.8, "stage_normal_rk32": 254.8}
FP64_LANES_PER_SM = 64

def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--id=%d" % self.index, "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for nm, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(self.rows), "reasons": sorted(reasons)}


def dist_setup(n_gpus):
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def bench_config(cfg, world):
    """The workload as both arms report it (the same dict)."""
    return {"workload": WORKLOAD, "grid": list(cfg["n"]), "ghost": 3, "cfl": cfg["cfl"],
            "reinit_interval": cfg["reinit_interval"], "reinit_iters": cfg["reinit_iters"],
            "seed": cfg["seed"],
            "l2": "inputs larger than L2 (144 MB per field)",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def sig(x, n=4):
    """Floats rounded to n significant digits, recursively."""
    if isinstance(x, float):
        return float("%.*g" % (n, x)) if np.isfinite(x) else x
    if isinstance(x, dict):
        return {k: sig(v, n) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [sig(v, n) for v in x]
    return x


# short names of nested keys in the final line's summaries
SHORT = {"error_vs_fp64.max_abs": "err_max", "error_vs_fp64.max_abs_band_5dx": "err_band5dx",
         "error_vs_fp64.l1_mean": "err_l1", "fd_check.max_rel_err": "fd_max_rel",
         "fd_check.max_err_over_max_grad": "fd_max_over_grad",
         "fd_check.max_rel_err_components_above_1pct": "fd_max_rel_above_1pct",
         "vs_initial.max_abs_band": "vs_phi0_band_max",
         "speedup_vs_per_grid_launches": "vs_per_grid_launches"}


def pick(d, *keys):
    """The keys of d that exist (dotted keys reach into nested dicts), under
    their short names."""
    if not isinstance(d, dict):
        return d
    out = {}
    for k in keys:
        cur, ok = d, True
        for part in k.split("."):
            if isinstance(cur, dict) and part in cur:
                cur = cur[part]
            else:
                ok = False
                break
        if ok:
            out[SHORT.get(k, k)] = cur
    return out


def run_parity(cfg, steps=2, reinit_pseudo_steps=1):
    """The timed configuration itself against the oracle: `steps` physical
    steps of the full 256^3 workload through the device drivers in the
    bench's arithmetic (FMA, single-reciprocal weights), then
    `reinit_pseudo_steps` reinitialization pseudo-steps, against the oracle's
    chain of the reference's routines in the reference integrators' order
    (LevelSetFunctionIntegrator.cc:1319-1510, ReinitializationAlgorithm.cc:
    177-330) over z-slab patches on all host cores.  Relative max-norm
    difference over the interior."""
    import oracle
    from lsmlib_b200 import gpu, integrator, workloads
    from oracle.driver import Grid, PatchedNormalStepper
    n = cfg["n"]
    gb, fb = workloads.boxes(n)
    dx = cfg["dx"]
    integrator.set_fp_mode(integrator.FP_FAST)
    ws = integrator.Workspace(gb, 8)
    d_phi = gpu.DeviceArray.from_host(cfg["phi"])
    d_F = gpu.DeviceArray.from_host(cfg["F"])
    ws.normal(d_phi, d_F, fb, dx, cfl=cfg["cfl"], nsteps=steps, step0=0,
              reinit_interval=10 ** 9, reinit_iters=0, use_phi0=cfg["use_phi0"])
    ws.reinit(d_phi, fb, dx, cfl=cfg["cfl"], iters=reinit_pseudo_steps,
              use_phi0=cfg["use_phi0"])
    got = d_phi.download()
    del ws, d_phi, d_F
    t0 = time.perf_counter()
    g = Grid(tuple(n), dx=dx)
    phi, F = g.field(cfg["phi"]), g.field(cfg["F"])
    ps = PatchedNormalStepper(oracle.oracle_toolbox(), g, os.cpu_count() or 1)
    parts, Fs = ps.scatter(phi), ps.scatter(F)
    for _ in range(steps):
        ps.normal_step(parts, Fs, cfg["cfl"])
    ps.reinit(parts, cfg["cfl"], reinit_pseudo_steps, cfg["use_phi0"])
    ps.gather(parts, phi)
    t_cpu = time.perf_counter() - t0
    want = g.interior(phi)
    have = g.interior(g.field(got))
    max_rel = float(np.max(np.abs(have - want)) / np.max(np.abs(want)))
    return {"max_rel": max_rel, "bound": 1e-12, "ok": max_rel <= 1e-12,
            "steps": steps, "reinit_pseudo_steps": reinit_pseudo_steps,
            "mode": "fast: FMA, one-reciprocal WENO5 weights",
            "oracle_s": round(t_cpu, 1)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local, pg):
    from lsmlib_b200 import gpu, integrator, workloads
    from lsmlib_b200.ext_abi import dbls, ints

    lib = gpu.load()
    gpu.check_rc(lib.lsmgpu_set_device(local), "set_device")
    cfg = workloads.config2(N_CELLS)
    n = cfg["n"]
    gb, fb = workloads.boxes(n)
    dx = cfg["dx"]
    cells = n[0] * n[1] * n[2]
    K, W = args.steps, args.warmup
    interval, iters = cfg["reinit_interval"], cfg["reinit_iters"]

    def run_steps(ws, d_phi, d_F, nsteps, step0):
        ws.normal(d_phi, d_F, fb, dx, cfl=cfg["cfl"], nsteps=nsteps, step0=step0,
                  reinit_interval=interval, reinit_iters=iters, use_phi0=cfg["use_phi0"])

    integrator.set_fp_mode(integrator.FP_FAST)
    timer = gpu.Timer()

    # ---- FP64, device resident -------------------------------------------
    ws = integrator.Workspace(gb, 8)
    d_phi = gpu.DeviceArray.from_host(cfg["phi"])
    d_F = gpu.DeviceArray.from_host(cfg["F"])
    run_steps(ws, d_phi, d_F, W, 0)
    gpu.check_rc(lib.lsmgpu_stream_synchronize(), "sync")
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    gpu.check_rc(lib.lsmgpu_stream_synchronize(), "sync")
    launches0 = lib.lsmgpu_kernel_launch_count()
    timer.start()
    run_steps(ws, d_phi, d_F, K, W)
    timer.stop()
    ms = timer.ms()
    gpu.check_rc(lib.lsmgpu_stream_synchronize(), "sync")
    launches = lib.lsmgpu_kernel_launch_count() - launches0
    barrier(pg)
    clk = clocks.stop()
    ms_max = max_over_ranks(pg, ms)
    value = world * cells * K / (ms_max / 1e3)
    phi64 = d_phi.download()

    # the two parts of a step separately: reinitialization pseudo-steps, and
    # physical steps without reinitialization
    timer.start()
    ws.reinit(d_phi, fb, dx, cfl=cfg["cfl"], iters=iters, use_phi0=cfg["use_phi0"])
    timer.stop()
    ms_re = max_over_ranks(pg, timer.ms())
    timer.start()
    ws.normal(d_phi, d_F, fb, dx, cfl=cfg["cfl"], nsteps=interval, step0=1,
              reinit_interval=10 ** 9, reinit_iters=0, use_phi0=cfg["use_phi0"])
    timer.stop()
    ms_no = max_over_ranks(pg, timer.ms())
    parts = {"reinit_pseudo_step": {"value": world * cells * iters / (ms_re / 1e3),
                                    "unit": "cell-updates/s",
                                    "ms_per_pseudo_step": ms_re / iters},
             "step_without_reinit": {"value": world * cells * interval / (ms_no / 1e3),
                                     "unit": UNIT, "ms_per_step": ms_no / interval}}

    fp32 = None
    if not args.no_fp32:
        # ---- FP32 form beside it -----------------------------------------
        ws32 = integrator.Workspace(gb, 4)
        d32 = gpu.DeviceArray.from_host(cfg["phi"].astype(np.float32))
        dF32 = gpu.DeviceArray.from_host(cfg["F"].astype(np.float32))
        run_steps(ws32, d32, dF32, W, 0)
        barrier(pg)
        gpu.check_rc(lib.lsmgpu_stream_synchronize(), "sync")
        timer.start()
        run_steps(ws32, d32, dF32, K, W)
        timer.stop()
        ms32 = max_over_ranks(pg, timer.ms())
        value32 = world * cells * K / (ms32 / 1e3)
        phi32 = d32.download().astype(np.float64)
        g = 3
        inner = (slice(g, g + n[0]), slice(g, g + n[1]), slice(g, g + n[2]))
        diff = np.abs(phi32[inner] - phi64[inner])
        band = np.abs(phi64[inner]) < 5 * dx[0]
        err32 = {"max_abs": float(diff.max()), "l1_mean": float(diff.mean()),
                 "max_abs_band_5dx": float(diff[band].max()) if band.any() else None,
                 "steps_compared": W + K}
        del d32, dF32, ws32
        fp32 = {"value": value32, "unit": UNIT, "ms_per_step": ms32 / K,
                "speedup_vs_fp64": value32 / value, "error_vs_fp64": err32,
                "policy": "FP32 phi and RHS, FP64 CFL reduction/dt/t, FP64 "
                          "reinitialization sign, stochastic rounding of stage outputs"}

    # ---- dominant kernels, timed alone on the same stream -----------------
    # the stage kernel the drivers launch: face-shared, two cells per
    # thread, reading ghost cells the drivers have stored (bc_mask 0 here:
    # phi64's ghost cells hold the drivers' last boundary values)
    peak, peak_kind = load_peaks()
    kern = {}
    for name, kind, rk, nbytes in (("stage_reinit_rk32", 2, 32, 3),
                                   ("stage_normal_rk32", 1, 32, 4)):
        # distinct stage input phi_s and RK base phi^n, as in the drivers
        a = gpu.DeviceArray(d_phi.shape)
        b = gpu.DeviceArray.from_host(phi64)
        c = gpu.DeviceArray.from_host(phi64)
        for _ in range(3):
            integrator.stage(kind, 8, a, b, c, [d_F], gb, fb, dx, 1e-3, rk, bc_mask=0)
        reps = 20
        timer.start()
        for _ in range(reps):
            integrator.stage(kind, 8, a, b, c, [d_F], gb, fb, dx, 1e-3, rk, bc_mask=0)
        timer.stop()
        t = timer.ms() / reps
        kern[name] = {"ms": t, "bytes": nbytes * 8 * cells}
        del a, b, c
    # launches per step at the reinit cadence: reinit 3*iters/interval,
    # normal 2 (+ the fused L/CFL pass)
    share_re = 3 * iters / interval * kern["stage_reinit_rk32"]["ms"]
    share_no = 3 * kern["stage_normal_rk32"]["ms"]
    dom = "stage_reinit_rk32" if share_re >= share_no else "stage_normal_rk32"
    achieved = kern[dom]["bytes"] / (kern[dom]["ms"] / 1e3) / 1e9
    traffic = NCU_TRAFFIC.get(dom) if N_CELLS == 256 else None
    # the FP64 pipe's share: the kernel's FP64 instructions per second over
    # the SMs' FP64 lanes at the SM clock sampled under load
    import torch
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    fp64_peak = n_sm * FP64_LANES_PER_SM * mhz * 1e6
    fp64_ach = NCU_FP64_OPS_PER_CELL[dom] * cells / (kern[dom]["ms"] / 1e3)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "traffic_source": "ncu capture, profiles/k_stage_pairs_config2_256.md",
                "fp64_pipe_active_pct_ncu": NCU_FP64_PIPE.get(dom),
                "fp64_frac": round(fp64_ach / fp64_peak, 3),
                "fp64": {"achieved_Tops": round(fp64_ach / 1e12, 2),
                         "peak_Tops": round(fp64_peak / 1e12, 2),
                         "ops_per_cell_ncu": NCU_FP64_OPS_PER_CELL[dom], "sms": n_sm,
                         "sm_mhz": mhz},
                "kernel": dom, "kernel_ms": round(kern[dom]["ms"], 4),
                "algorithmic_bytes_per_launch": kern[dom]["bytes"],
                "peak_source": peak_kind,
                "other_kernels": {k: round(v["ms"], 4) for k, v in kern.items() if k != dom}}

    e2e = None
    if not args.no_e2e:
        # ---- e2e: host-resident level set through the C ABI ----------------
        h_phi = lib.lsmgpu_host_alloc(cfg["phi"].nbytes)
        h_F = lib.lsmgpu_host_alloc(cfg["F"].nbytes)
        count = cfg["phi"].size
        hp = np.ctypeslib.as_array((ctypes.c_double * count).from_address(h_phi))
        hf = np.ctypeslib.as_array((ctypes.c_double * count).from_address(h_F))
        hp[:] = cfg["phi"].ravel(order="F")
        hf[:] = cfg["F"].ravel(order="F")
        ws_e = integrator.Workspace(gb, 8)
        nb = cfg["phi"].nbytes

        def e2e_step(s):
            # one step per call on the host arrays: phi and F copied in, phi
            # copied back (slab-pipelined inside the call)
            ws_e.normal_host(h_phi, h_F, fb, dx, cfl=cfg["cfl"], nsteps=1, step0=s,
                             reinit_interval=interval, reinit_iters=iters,
                             use_phi0=cfg["use_phi0"])

        def e2e_run(async_on):
            ws_e.set_host_async(async_on)
            for s in range(W):
                e2e_step(s)
            ws_e.sync()
            barrier(pg)
            t0 = time.perf_counter()
            for s in range(W, W + K):
                e2e_step(s)
            ws_e.sync()     # the last step's phi is back in host memory
            return max_over_ranks(pg, time.perf_counter() - t0)

        t_block = e2e_run(False)
        hp[:] = cfg["phi"].ravel(order="F")
        t_e2e = e2e_run(True)
        e2e = {"value": world * cells * K / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": 2 * nb, "d2h_bytes_per_step": nb,
               "ms_per_step": 1e3 * t_e2e / K,
               "blocking_ms_per_step": 1e3 * t_block / K,
               "path": "lsmgpu_normal_tvdrk3_host, one call per step on phi and F "
                       "in pinned host memory: both copied in and phi copied back "
                       "every step in z-slabs; calls queued on the workspace "
                       "(lsmgpu_workspace_set_host_async), the speed double-"
                       "buffered, each slab copied in once the previous call's "
                       "copy of it back has landed; timer stopped after "
                       "lsmgpu_workspace_sync"}
        lib.lsmgpu_host_free(h_phi)
        lib.lsmgpu_host_free(h_F)

    batched_res = None
    if not args.no_batched:
        batched_res = run_batched(lib, pg, world)
        if rank == 0 and world == 1 and not args.no_cpu:
            batched_res["cpu_baseline"] = cpu_batched_sample()

    adjoint_res = None
    if not args.no_adjoint:
        adjoint_res = run_adjoint()

    toolbox_res = None
    if not args.no_toolbox:
        toolbox_res = run_toolbox(peak)

    distance_res = None
    if not args.no_distance:
        distance_res = run_distance()

    deformation_res = None
    if not args.no_deformation:
        deformation_res = run_config3(lib, pg, world,
                                      n_full=512 if args.config3_full else 256)

    parity = None
    if rank == 0 and not args.no_parity:
        parity = run_parity(cfg)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(cfg)

    # every leg in full on a line of its own; the final line carries compact
    # summaries (the driver keeps the last few KB of the output)
    legs = {"parts": parts, "fp32": fp32, "batched": batched_res, "adjoint": adjoint_res,
            "deformation": deformation_res, "toolbox": toolbox_res,
            "distance": distance_res, "roofline": roofline, "e2e": e2e, "parity": parity,
            "cpu_baseline": cpu}
    if rank == 0:
        for k, v in legs.items():
            if v is not None:
                print(json.dumps({"bench_detail": k, "data": v}), flush=True)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": bench_config(cfg, world),
        "parts": {k: sig(pick(v, "value", "ms_per_pseudo_step", "ms_per_step"))
                  for k, v in parts.items()},
        "parity": sig(pick(parity, "max_rel", "bound", "ok", "steps", "reinit_pseudo_steps",
                           "mode"), 3) if parity else None,
        "fp32": sig(pick(fp32, "value", "speedup_vs_fp64", "error_vs_fp64.max_abs",
                         "error_vs_fp64.max_abs_band_5dx", "error_vs_fp64.l1_mean")),
        "batched": sig(compact_batched(batched_res)),
        "adjoint": sig(pick(adjoint_res, "reverse_over_forward", "gradient_over_forward",
                            "forward_ms", "reverse_ms", "fd_check.max_rel_err",
                            "fd_check.max_rel_err_components_above_1pct")),
        "deformation": sig(compact_deformation(deformation_res), 3),
        "toolbox": sig(compact_toolbox(toolbox_res)),
        "distance": sig(compact_distance(distance_res)),
        "roofline": sig(pick(roofline, "bound", "achieved", "peak", "unit", "frac",
                             "traffic", "kernel", "kernel_ms", "peak_source",
                             "fp64_pipe_active_pct_ncu", "fp64_frac")),
        "e2e": sig(pick(e2e, "value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step",
                        "ms_per_step", "blocking_ms_per_step")),
        "gpu_launches": int(launches),
        "clocks": sig(clk),
    }
    if cpu is not None:
        line["cpu_baseline"] = sig(pick(cpu, "value", "unit", "cores", "kind", "sample"))
        line["cpu_baseline"]["sample"] = "256x256x64 slab, 1 step + its reinit share"
    return line


def compact_batched(r):
    if not r:
        return r
    out = {"cells": r.get("cells")}
    for key in ("fp64", "fp32"):
        e = r.get(key) or {}
        out[key] = pick(e, "value", "speedup_vs_per_grid_launches",
                        "error_vs_fp64.max_abs", "error_vs_fp64.max_abs_band_5dx")
    if "cpu_baseline" in r:
        out["cpu"] = pick(r["cpu_baseline"], "value", "cores")
    return out


def compact_deformation(r):
    """Throughput of each form, the FP64 reversal's error against the initial
    interface (the FP32 forms' equals it to the digits shown) and the FP32
    forms' errors against FP64 (the full entries are on the detail line)."""
    if not r:
        return r
    out = {}
    for k, v in r.items():
        if not isinstance(v, dict):
            continue
        keys = ["value", "error_vs_fp64.max_abs", "error_vs_fp64.max_abs_band_5dx"]
        if k.startswith("reversal") and k.endswith("fp64"):
            keys.append("vs_initial.max_abs_band")
        out[k] = pick(v, *keys)
    return out


def compact_toolbox(r):
    """Routine count and the spread of their HBM fractions (the per-routine
    table is on its detail line)."""
    if not r:
        return r
    r = r.get("routines", r)
    fr = sorted(v["frac_of_measured_hbm"] for v in r.values()
                if isinstance(v, dict) and "frac_of_measured_hbm" in v)
    if not fr:
        return {"routines": len(r)}
    return {"routines": len(fr), "hbm_frac_min": fr[0], "hbm_frac_median": fr[len(fr) // 2],
            "hbm_frac_max": fr[-1]}


def compact_distance(r):
    """Points/s of each solver and order at the largest grid, and whether
    every result checked against the oracle was bit-exact (the full table is
    on its detail line)."""
    if not r or "sizes" not in r:
        return r
    sizes = r["sizes"]
    big = max(sizes, key=lambda k: int(k.split("^")[0]))
    pts = {k: v["value"] for k, v in sizes[big].items() if isinstance(v, dict) and "value" in v}
    exact = [v["bitwise_vs_oracle"] for e in sizes.values() for v in e.values()
             if isinstance(v, dict) and "bitwise_vs_oracle" in v]
    return {"grid": big, "points_per_s": pts,
            "bit_exact_all_checked": all(exact) if exact else None}


def run_adjoint(n_fd=20, h=2e-5):
    """Config 5: 128^3, B-spline velocity (8^3 x 3 coefficients), 200 steps,
    checkpoints every 15 steps.  Times the forward run (with its
    checkpoints) and the reverse sweep (segment recomputation included), and
    checks dJ/dtheta against central finite differences of the GPU forward
    model on n_fd seeded coefficients.  The forward map is smooth only
    piecewise (upwind side, eps argmax and the kinks of H_eps''), so the
    difference quotients scatter at the 1e-6 level below h ~ 1e-5 and grow
    as O(h^2) above it; h = 2e-5 sits between the two."""
    from lsmlib_b200 import adjoint, workloads
    cfg = workloads.config5()
    p = adjoint.AdvectionAdjoint(cfg["n"], cfg["dx"], cfg["x_lo"], cfg["lattice"],
                                 cfg["steps"], 15)
    p.set_theta(cfg["theta"])
    dt = p.cfl_dt(cfg["cfl"])
    p.set_dt(dt)
    p.set_fields(cfg["phi0"], cfg["target"], cfg["eps"])
    p.forward()
    p.backward()                        # warm-up
    fwd, rev = [], []
    for _ in range(3):
        loss = p.forward()
        f, _ = p.timing()
        gt, gp = p.backward()
        _, a = p.timing()
        fwd.append(f)
        rev.append(a)
    f, a = min(fwd), min(rev)
    rng = np.random.default_rng(cfg["seed"])
    picks = rng.choice(gt.size, n_fd, replace=False)
    theta = cfg["theta"]
    worst = worst_abs = worst_sig = 0.0
    scale = float(np.max(np.abs(gt)))
    inner = tuple(slice(3, 3 + v) for v in cfg["n"])
    target = np.asarray(cfg["target"])[inner]
    vol = float(np.prod(cfg["dx"]))

    def final(t):
        p.set_theta(t)
        p.forward()
        return p.phi_final()[inner]

    for q in picks:
        idx = np.unravel_index(q, gt.shape)
        t = theta.copy()
        t[idx] += h
        fa = final(t)
        t[idx] -= 2 * h
        fb = final(t)
        fd = adjoint.loss_difference(fa, fb, target, cfg["eps"], vol) / (2 * h)
        worst = max(worst, abs(fd - gt[idx]) / max(abs(fd), 1e-3 * scale))
        worst_abs = max(worst_abs, abs(fd - gt[idx]) / scale)
        if abs(fd) >= 1e-2 * scale:
            worst_sig = max(worst_sig, abs(fd - gt[idx]) / abs(fd))
    p.close()
    cells = cfg["n"][0] * cfg["n"][1] * cfg["n"][2]
    return {"workload": "128^3, trilinear B-spline velocity on 8^3 x 3 coefficients, "
                        "sphere to ellipsoid, WENO5 + TVD-RK3, 200 steps, frozen dt, "
                        "checkpoints every 15 steps",
            "loss": loss, "dt": dt, "forward_ms": f, "reverse_ms": a,
            "reverse_over_forward": a / f, "gradient_over_forward": (f + a) / f,
            "forward_cell_updates_per_s": cells * cfg["steps"] / (f / 1e3),
            "fd_check": {"coefficients": n_fd, "h": h,
                         "max_rel_err": worst,
                         "rel_err_floor": "1e-3 * max|dJ/dtheta|",
                         "max_err_over_max_grad": worst_abs,
                         "max_rel_err_components_above_1pct": worst_sig,
                         "loss_difference": "cell by cell from the two final states"}}


# drop-in routines timed one by one on the 256^3 grid with device arrays
TOOLBOX_TIMED = [
    "lsm3dhjweno5_", "lsm3dupwindhjweno5_", "lsm3dhjeno3_", "lsm3daddnormalveltermtolserhs_",
    "lsm3dcomputereinitializationeqnrhs_", "lsm3dtvdrk3stage3_",
    "lsm3dcomputestablenormalveldt_", "lsm3dcentralgradorder2_", "lsm3dcentralgradorder4_",
    "lsm3dlaplacianorder2_", "lsm3dphiupwindgradf_", "lsm3daveragegradphi_",
    "lsm3dgradientmagnitude_", "lsm3daddconstcurvtermtolserhs_",
    "lsm3daddconstprecomputedcurvtermtolserhs_", "lsm3daddexternalandnormalveltermtolserhs_",
    "lsm3dcomputeorthogonalizationeqnrhs_", "lsm3dcomputedistanceforsubcellfix_",
    "lsm3dcomputereinitializationeqnrhssubcellfixorder1_"]


def run_toolbox(peak, n=256, reps=10):
    """Each routine of TOOLBOX_TIMED through the C ABI on device arrays over
    the n^3 fill box (FP64, reference expression order): mean device time of
    `reps` calls and the algorithmic bytes over the fill box (each input
    array read once, each output written once, in/out arrays both)."""
    from lsmlib_b200 import abi, gpu, workloads
    from lsmlib_b200.toolbox import Field
    tb = gpu.toolbox()
    cfg = workloads.config2(n)
    gb, fb = workloads.boxes(cfg["n"])
    lo = (gb[0], gb[2], gb[4])
    shape = cfg["phi"].shape
    rng = np.random.default_rng(7)
    # every array of a call is its own 144 MB buffer (larger than L2), so no
    # input is served from L2 on behalf of another
    noise = np.asfortranarray(rng.standard_normal(shape))
    ins = [gpu.DeviceArray.from_host(noise) for _ in range(14)]   # [-1]: scratch
    level_set = gpu.DeviceArray.from_host(cfg["phi"])
    pool = [gpu.DeviceArray.from_host(noise) for _ in range(6)]
    # subcell fix: every cell away from the interface (the far-field flag
    # -1000 max dx), so the Godunov branch reads all gradient arrays
    far = gpu.DeviceArray.from_host(np.full(shape, -1000.0 * max(cfg["dx"]), order="F"))
    cells = n ** 3
    timer = gpu.Timer()
    res = {}
    for sym in TOOLBOX_TIMED:
        fields, scal, nbytes, k_out, k_in = {}, {}, 0, 0, 0
        for kind, name in abi.parse(abi.SIGNATURES[sym]):
            if kind == "S":
                fields[name] = Field(ins[-1], lo)     # scratch, never touched
            elif kind == "I":
                if name == "distance0":
                    d = far
                elif name in ("phi", "phi0", "u_cur") and level_set not in [
                        f.data for f in fields.values()]:
                    d = level_set
                else:
                    d = ins[k_in]
                    k_in += 1
                fields[name] = Field(d, lo)
                nbytes += 8 * cells
            elif kind in ("O", "X"):
                fields[name] = Field(pool[k_out], lo)
                k_out += 1
                nbytes += (2 if kind == "X" else 1) * 8 * cells
            elif kind == "R":
                scal[name] = {"dx": cfg["dx"][0], "dy": cfg["dx"][1], "dz": cfg["dx"][2],
                              "dt": 1e-3, "cfl_number": 0.5, "vel_n": 0.8, "b": 0.1}[name]
            elif kind == "N":
                scal[name] = 0
        for _ in range(2):
            tb.call(sym, fields, fb, **scal)
        timer.start()
        for _ in range(reps):
            tb.call(sym, fields, fb, **scal)
        timer.stop()
        ms = timer.ms() / reps
        gbs = nbytes / (ms / 1e3) / 1e9
        res[sym] = {"ms": round(ms, 4), "algorithmic_bytes": nbytes,
                    "gb_s": round(gbs, 1), "frac_of_measured_hbm": round(gbs / peak, 3)}
    return {"grid": "256^3 fill box, 262^3 ghost boxes, FP64, device arrays, mean of "
                    "%d calls" % reps, "routines": res}


def run_distance(n=256, n_cpu=128, reps=3):
    """The fast marching routines on workloads.distance_case at n^3 and
    n_cpu^3, orders 1 and 2: the signed distance function
    (computeDistanceFunction3d), three extension fields
    (computeExtensionFields3d) and the Eikonal solution
    (solveEikonalEquation3d, the region phi <= 0 as boundary data).  Device
    arrays timed with CUDA events (mean of ``reps`` solves), the drop-in entry
    point on host arrays (copies included), and at n_cpu^3 the CPU oracle
    (the reference's heap march restated in C, one core) with a bit-for-bit
    comparison."""
    import oracle
    from lsmlib_b200 import gpu, workloads
    lib = gpu.load()
    P = ctypes.c_void_p
    drop_in = {"distance": lib.computeDistanceFunction3d,
               "extension": lib.computeExtensionFields3d,
               "eikonal": lib.solveEikonalEquation3d}
    drop_in["distance"].argtypes = [P] * 3 + [ctypes.c_int, P, P]
    drop_in["extension"].argtypes = [P] * 6 + [ctypes.c_int, ctypes.c_int, P, P]
    drop_in["eikonal"].argtypes = [P] * 3 + [ctypes.c_int, P, P]
    for f in drop_in.values():
        f.restype = ctypes.c_int
    timer = gpu.Timer()
    out = {"workload": "config-2 union of 6 spheres on [-1,1]^3, scaled by "
                       "1.2 + 0.5 sin(3 pi x) sin(2 pi y) cos(pi z) (same zero set); "
                       "extension: 3 source fields; eikonal: phi <= 0 (shifted by "
                       "-min phi) as boundary data, speed 1 + 0.5 sin(6x) cos(4y)",
           "unit": "grid points/s", "sizes": {}}
    for size in (n_cpu, n):
        phi, dx = workloads.distance_case(size)
        a = np.linspace(-1.0, 1.0, size)
        srcs = [np.asfortranarray(np.broadcast_to(v, phi.shape)) for v in
                (a[:, None, None] + 0 * a[None, :, None],
                 np.sin(3 * a)[None, :, None] + 0 * a[:, None, None],
                 np.cos(2 * a)[None, None, :] + 0 * a[:, None, None])]
        speed = np.asfortranarray(1.0 + 0.5 * np.sin(6 * a)[:, None, None] *
                                  np.cos(4 * a)[None, :, None] + 0 * a[None, None, :])
        minphi = phi.min()
        eik_data = np.asfortranarray(np.where(phi > 0, minphi - 1.0, phi) - minphi)
        pts = size ** 3
        d_phi = gpu.DeviceArray.from_host(phi)
        d_out = gpu.DeviceArray(phi.shape)
        d_src = [gpu.DeviceArray.from_host(x) for x in srcs]
        d_ext = [gpu.DeviceArray(phi.shape) for _ in srcs]
        d_speed = gpu.DeviceArray.from_host(speed)
        d_eik0 = gpu.DeviceArray.from_host(eik_data)
        dims = (ctypes.c_int * 3)(size, size, size)
        h = (ctypes.c_double * 3)(*dx)
        hd = np.ascontiguousarray(np.array(dx))
        hdims = np.array([size] * 3, dtype=np.intc)
        ext_p = (ctypes.c_void_p * 3)(*[x.ptr for x in d_ext])
        src_p = (ctypes.c_void_p * 3)(*[x.ptr for x in d_src])
        entry = {}
        for solver in ("distance", "extension", "eikonal"):
            for order in (1, 2):
                passes = ctypes.c_int(0)

                def device_solve(pp=None):
                    # the Eikonal solver overwrites its boundary data: restore it
                    # (outside the timed region)
                    if solver == "eikonal":
                        lib.lsmgpu_memcpy_dtod(d_out.ptr, d_eik0.ptr, d_out.nbytes)
                    timer.start()
                    if solver == "distance":
                        rc = lib.lsmgpu_distance_function3d(d_out.ptr, d_phi.ptr, None, order,
                                                            dims, h, pp)
                    elif solver == "extension":
                        rc = lib.lsmgpu_extension_fields3d(d_out.ptr, ctypes.cast(ext_p, P),
                                                           d_phi.ptr, None,
                                                           ctypes.cast(src_p, P), None, 3,
                                                           order, dims, h, pp)
                    else:
                        rc = lib.lsmgpu_eikonal3d(d_out.ptr, d_speed.ptr, None, order, dims, h,
                                                  pp)
                    timer.stop()
                    return rc, timer.ms()
                gpu.check_rc(device_solve(ctypes.byref(passes))[0], solver)
                ms = sum(device_solve()[1] for _ in range(reps)) / reps
                # the drop-in entry point on host arrays
                host = np.zeros_like(phi)
                hext = [np.zeros_like(phi) for _ in srcs]
                hext_p = (ctypes.c_void_p * 3)(*[x.ctypes.data for x in hext])
                hsrc_p = (ctypes.c_void_p * 3)(*[x.ctypes.data for x in srcs])
                t_e2e = float("inf")
                for _ in range(2):      # best of two: the first may grow the memory pool
                    if solver == "eikonal":
                        host[...] = eik_data
                    t0 = time.perf_counter()
                    if solver == "distance":
                        rc = drop_in[solver](host.ctypes.data, phi.ctypes.data, None, order,
                                             hdims.ctypes.data, hd.ctypes.data)
                    elif solver == "extension":
                        rc = drop_in[solver](host.ctypes.data, ctypes.cast(hext_p, P),
                                             phi.ctypes.data, None, ctypes.cast(hsrc_p, P),
                                             None, 3, order, hdims.ctypes.data, hd.ctypes.data)
                    else:
                        rc = drop_in[solver](host.ctypes.data, speed.ctypes.data, None, order,
                                             hdims.ctypes.data, hd.ctypes.data)
                    t_e2e = min(t_e2e, time.perf_counter() - t0)
                r = {"ms": round(ms, 2), "value": pts / (ms / 1e3), "passes": passes.value,
                     "e2e": {"ms": round(1e3 * t_e2e, 2), "value": pts / t_e2e, "rc": rc,
                             "path": "the reference's entry point on host arrays (copies "
                                     "included), best of 2 calls"}}
                if size == n_cpu:
                    t0 = time.perf_counter()
                    if solver == "distance":
                        want = [oracle.oracle_fmm(ordered=True)(phi.T, order, dx)]
                    elif solver == "extension":
                        dist, fields = oracle.oracle_extension(ordered=True)(phi.T, [x.T for x in srcs],
                                                                 order, dx)
                        want = [dist] + fields
                    else:
                        want = [oracle.oracle_eikonal(ordered=True)(eik_data.T, speed.T, order, dx)]
                    t_cpu = time.perf_counter() - t0
                    got = [host.T] + ([x.T for x in hext] if solver == "extension" else [])
                    r["cpu_oracle"] = {"ms": round(1e3 * t_cpu, 1), "value": pts / t_cpu,
                                       "cores": 1, "kind": "port"}
                    r["bitwise_vs_oracle"] = all(
                        np.array_equal(np.ascontiguousarray(x).view(np.uint64),
                                       np.ascontiguousarray(y).view(np.uint64))
                        for x, y in zip(got, want))
                entry["%s_order%d" % (solver, order)] = r
        out["sizes"]["%d^3" % size] = entry
        for x in [d_phi, d_out, d_speed, d_eik0] + d_src + d_ext:
            x.free()
    return out


def deformation_run(ws, d_phi, fb, cfg, timer):
    """Advance to t_end in chunks sized from the last dt (the driver clips
    the final dt at t_end, so no step is taken past it); device time and
    step count."""
    from lsmlib_b200 import gpu
    t_end, ms, steps, chunk = cfg["t_end"], 0.0, 0, 16
    while True:
        timer.start()
        ws.deformation(d_phi, fb, cfg["dx"], cfg["x_lo"], period=cfg["period"],
                       cfl=cfg["cfl"], t_end=t_end, nsteps=chunk)
        timer.stop()
        ms += timer.ms()
        steps += chunk
        t, dt = ws.time()
        left = t_end - t
        if left <= 1e-13 * t_end:
            return ms, steps, t
        chunk = max(1, min(2048, int(0.9 * left / max(dt, 1e-300))))


def interface_errors(phi, ref, dx, band_dx=3):
    """max and mean |phi - ref| in the band |ref| < band_dx dx, and the relative
    change of the enclosed volume sum H(-phi) dx^3 (LSM_HEAVISIDE, eps 1.5 dx)."""
    from lsmlib_b200.adjoint import heaviside
    band = np.abs(ref) < band_dx * dx
    d = np.abs(phi - ref)
    v = float(np.sum(heaviside(-phi, 1.5 * dx)))
    v0 = float(np.sum(heaviside(-ref, 1.5 * dx)))
    return {"max_abs_band": float(d[band].max()), "mean_abs_band": float(d[band].mean()),
            "band": "|phi0| < %d dx" % band_dx, "volume_rel_change": (v - v0) / v0}


def run_config3(lib, pg, world, n_window=512, window=100, n_full=256):
    """Config 3: LeVeque's deformation of a sphere (r 0.15 at (0.35,0.35,0.35)
    on [0,1]^3, period 3) by WENO5 + TVD-RK3 at CFL 0.5, velocity evaluated
    in the stage kernels.  Throughput of FP64 and FP32 over the first
    `window` steps at n_window^3; the full reversal to t = 3 at n_full^3 with
    the errors against the initial interface and FP32 against FP64."""
    from lsmlib_b200 import gpu, integrator, workloads
    timer = gpu.Timer()
    res = {"workload": "LeVeque deformation of a sphere, period 3, WENO5 + TVD-RK3, "
                       "CFL 0.5, velocity in-kernel (no velocity arrays)"}
    # the FP32 form as it is, and with the tiles near the interface in FP64
    # (FP64_BAND: |phi| < 16 dx, widened by one tile)
    forms = ((8, "fp64", 0), (4, "fp32", 0), (4, "fp32band", integrator.FP64_BAND))
    cfg = workloads.config3(n_window)
    gb, fb = workloads.boxes(cfg["n"])
    cells = cfg["n"][0] * cfg["n"][1] * cfg["n"][2]
    for prec, key, extra in forms:
        dtype = np.float64 if prec == 8 else np.float32
        ws = integrator.Workspace(gb, prec)
        if extra:
            ws.set_fp64_policy(integrator.FP64_SIGN | integrator.STOCH_ROUND | extra)
        d = gpu.DeviceArray.from_host(cfg["phi"].astype(dtype))
        ws.deformation(d, fb, cfg["dx"], cfg["x_lo"], period=cfg["period"], cfl=cfg["cfl"],
                       t_end=cfg["t_end"], nsteps=3)
        barrier(pg)
        timer.start()
        ws.deformation(d, fb, cfg["dx"], cfg["x_lo"], period=cfg["period"], cfl=cfg["cfl"],
                       t_end=cfg["t_end"], nsteps=window)
        timer.stop()
        ms = max_over_ranks(pg, timer.ms())
        res["window_%d_%s" % (n_window, key)] = {
            "value": world * cells * window / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / window, "steps": window}
        del d, ws
    cfg = workloads.config3(n_full)
    gb, fb = workloads.boxes(cfg["n"])
    inner = tuple(slice(3, 3 + v) for v in cfg["n"])
    phi0 = cfg["phi"][inner]
    finals = {}
    for prec, key, extra in forms:
        dtype = np.float64 if prec == 8 else np.float32
        ws = integrator.Workspace(gb, prec)
        if extra:
            ws.set_fp64_policy(integrator.FP64_SIGN | integrator.STOCH_ROUND | extra)
        d = gpu.DeviceArray.from_host(cfg["phi"].astype(dtype))
        ms, steps, t = deformation_run(ws, d, fb, cfg, timer)
        finals[key] = d.download()[inner].astype(np.float64)
        res["reversal_%d_%s" % (n_full, key)] = dict(
            {"steps": steps, "t": t, "ms": ms,
             "value": n_full ** 3 * steps / (ms / 1e3), "unit": UNIT},
            vs_initial=interface_errors(finals[key], phi0, cfg["dx"][0]))
        del d, ws
    band = np.abs(finals["fp64"]) < 5 * cfg["dx"][0]
    for key in ("fp32", "fp32band"):
        diff = np.abs(finals[key] - finals["fp64"])
        res["reversal_%d_%s" % (n_full, key)]["error_vs_fp64"] = {
            "max_abs": float(diff.max()), "l1_mean": float(diff.mean()),
            "max_abs_band_5dx": float(diff[band].max())}
    return res


def run_batched(lib, pg, world, steps=50, warmup=3):
    """Config 4: 256 grids of U{32..128}^3 cells, constant velocities, own CFL
    dt, 50 TVD-RK3 steps; FP64 and FP32 through one persistent work-list
    launch per stage replayed from a CUDA graph (autotuned tile), and FP64
    through one launch per grid per stage for comparison."""
    from lsmlib_b200 import batched, gpu, workloads
    cfg = workloads.config4()
    res = {"workload": "256 grids, per-axis U{32..128}, 1-8 spheres, constant "
                       "velocity U(-1,1)^3, WENO5 + TVD-RK3, CFL 0.5, 50 steps, "
                       "periodic boundaries",
           "grids": len(cfg["sizes"]), "steps": steps}
    timer = gpu.Timer()
    finals = {}
    for prec, key in ((8, "fp64"), (4, "fp32")):
        dtype = np.float64 if prec == 8 else np.float32
        b = batched.Batch(cfg["sizes"], cfg["dx"], prec)
        b.upload(workloads.config4_phi(cfg, dtype))
        b.set_velocity(cfg["vel"], cfg["cfl"])
        b.set_bc(batched.BC_PERIODIC)
        res["cells"] = int(b.cells)
        tune = b.autotune(report=True)
        shape, tile = b.tile()
        gpu.check_rc(lib.lsmgpu_set_stream(b.stream()), "set_stream")
        b.advect(warmup, batched.MODE_GRAPH)
        barrier(pg)
        timer.start()
        b.advect(steps, batched.MODE_GRAPH, sync=False)
        timer.stop()
        ms = max_over_ranks(pg, timer.ms())
        finals[key] = [a[3:-3, 3:-3, 3:-3].astype(np.float64) for a in b.download()]
        entry = {"value": world * b.cells * steps / (ms / 1e3), "unit": UNIT,
                 "ms_per_step": ms / steps, "tile": list(tile),
                 "autotune_ms_per_step": [round(t, 4) for t in tune]}
        if prec == 8:
            # the plain path: one launch per grid per stage, same kernels
            b2 = batched.Batch(cfg["sizes"], cfg["dx"], prec)
            b2.upload(workloads.config4_phi(cfg, dtype))
            b2.set_velocity(cfg["vel"], cfg["cfl"])
            b2.set_bc(batched.BC_PERIODIC)
            b2.set_tile(shape)
            gpu.check_rc(lib.lsmgpu_set_stream(b2.stream()), "set_stream")
            b2.advect(warmup, batched.MODE_PER_GRID)
            timer.start()
            b2.advect(steps, batched.MODE_PER_GRID, sync=False)
            timer.stop()
            ms2 = max_over_ranks(pg, timer.ms())
            entry["per_grid_launches_value"] = world * b2.cells * steps / (ms2 / 1e3)
            entry["speedup_vs_per_grid_launches"] = ms2 / ms
            b2.close()
        res[key] = entry
        gpu.check_rc(lib.lsmgpu_set_stream(None), "set_stream")
        b.close()
    d = [np.abs(a - b) for a, b in zip(finals["fp32"], finals["fp64"])]
    band = [np.abs(b) < 5 * max(dx) for b, dx in zip(finals["fp64"], cfg["dx"])]
    flat = np.concatenate([x.ravel() for x in d])
    res["fp32"]["error_vs_fp64"] = {
        "max_abs": float(flat.max()), "l1_mean": float(flat.mean()),
        "max_abs_band_5dx": float(max(x[m].max() for x, m in zip(d, band) if m.any())),
        "steps_compared": warmup + steps}
    res["fp32"]["policy"] = "FP32 phi, FP64 per-grid dt, stochastic rounding of stage outputs"
    return res


# ---------------------------------------------------------------------------
# CPU reference
# ---------------------------------------------------------------------------
def slab_case(cfg, nz):
    """A z-slab of the config-2 grid: rows through the middle of the domain,
    linear-extrapolation boundaries on all faces of the slab."""
    from oracle.driver import Grid
    n = cfg["n"]
    k0 = (n[2] - nz) // 2
    g = Grid((n[0], n[1], nz), dx=cfg["dx"])
    ks = slice(k0, k0 + nz + 6)
    phi = g.field(cfg["phi"][:, :, ks])
    F = g.field(cfg["F"][:, :, ks])
    return g, phi, F


def reference_toolbox():
    import oracle
    if oracle.reference_available():
        return oracle.reference_toolbox(), "reference"
    return oracle.oracle_toolbox(), "port"


def cpu_baseline_sample(cfg, nz=64):
    """Single-thread reference routines on a 256x256xnz slab: one normal step
    and two reinitialization pseudo-steps (the per-step share of 20
    pseudo-steps every 10 steps)."""
    from oracle.driver import Stepper
    tb, kind = reference_toolbox()
    g, phi, F = slab_case(cfg, nz)
    st = Stepper(tb, g)
    t0 = time.perf_counter()
    st.normal_step(phi, F, cfg["cfl"])
    t1 = time.perf_counter()
    st.reinit(phi, cfg["cfl"], 2)
    t2 = time.perf_counter()
    per_step = (t1 - t0) + (t2 - t1) * (cfg["reinit_iters"] / cfg["reinit_interval"]) / 2
    cells = g.n[0] * g.n[1] * g.n[2]
    return {"value": cells / per_step, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": "256x256x%d slab of the workload: 1 step + 2 reinit pseudo-steps "
                      "(= the reinit share of one step), %.1f s" % (nz, t2 - t0)}


_C4_TOOLBOX = None


def _c4_step(i):
    """One external-velocity TVD-RK3 step of config-4 grid ``i`` with the
    reference's routines (a process-pool task): (cells, seconds)."""
    global _C4_TOOLBOX
    from oracle.driver import Grid, Stepper
    from lsmlib_b200 import workloads
    if _C4_TOOLBOX is None:
        _C4_TOOLBOX = reference_toolbox()[0]
    cfg = workloads.config4()
    n, dx, vel = cfg["sizes"][i], cfg["dx"][i], cfg["vel"][i]
    ax, centres, radii = cfg["grids"][i]
    g = Grid(n, dx=dx)
    phi = g.field(workloads.union_of_spheres(ax, centres, radii))
    v = [g.field(np.full(g.shape, c, order="F")) for c in vel]
    st = Stepper(_C4_TOOLBOX, g, bc="periodic")
    t0 = time.perf_counter()
    dt = st.advect_dt(v, cfg["cfl"])
    st.advect_step(phi, lambda c: v, dt)
    return n[0] * n[1] * n[2], time.perf_counter() - t0


def cpu_batched_sample():
    """Config 4 on all host cores: independent grids, one process each, the
    reference's routines; one step of each of the first 4 x cores grids."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    grids = list(range(min(256, 4 * cores)))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_c4_step, range(cores))          # start-up and first-touch
        t0 = time.perf_counter()
        res = pool.map(_c4_step, grids)
        wall = time.perf_counter() - t0
    cells = sum(c for c, _ in res)
    return {"value": cells / wall, "unit": UNIT, "cores": cores,
            "kind": reference_toolbox()[1],
            "sample": "one TVD-RK3 step of each of the first %d config-4 grids (%.1f M "
                      "cells), one process per core, %.1f s" % (len(grids), cells / 1e6, wall)}


def run_reference(args, world, rank, budget_s=90.0):
    """The reference's own toolbox routines (the translated Fortran when it
    is built, else the C oracle) on the same workload as our arm: the full
    256^3 grid, patch-decomposed in z with one patch per host thread (16
    patches of 16 planes on a 16-core host), as the reference's parallel
    package runs it -- a 3-cell ghost exchange before every stage and the
    minimum of the patch dts (LevelSetFunctionIntegrator.cc:382, :567,
    :1377).  A step is one time step plus its share of reinitialization
    (2 pseudo-steps: 20 every 10 steps).  The warm-up steps run in full; the
    timed steps stop once `budget_s` seconds have passed (the rate is the
    same per step), so the run stays within a few minutes."""
    if rank != 0:
        return None
    from oracle.driver import Grid, PatchedNormalStepper
    from lsmlib_b200 import workloads
    cfg = workloads.config2(N_CELLS)
    threads = os.cpu_count() or 1
    tb, kind = reference_toolbox()
    g = Grid(tuple(cfg["n"]), dx=cfg["dx"])
    ps = PatchedNormalStepper(tb, g, threads)
    parts, Fs = ps.scatter(g.field(cfg["phi"])), ps.scatter(g.field(cfg["F"]))
    iters_per_step = cfg["reinit_iters"] // cfg["reinit_interval"]

    def step():
        ps.normal_step(parts, Fs, cfg["cfl"])
        ps.reinit(parts, cfg["cfl"], iters_per_step, cfg["use_phi0"])

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    timed = 0
    while timed < args.steps:
        step()
        timed += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    cells = g.n[0] * g.n[1] * g.n[2]
    value = cells * timed / dt
    planes = sorted({pg.n[2] for pg, _ in ps.patches})
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": bench_config(cfg, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": "full %s grid, %d z-patches of %s planes on %d threads; "
                                   "%d of %d steps timed (%.0f s budget); a step = 1 time "
                                   "step + %d reinit pseudo-steps"
                                   % ("x".join(map(str, cfg["n"])), len(ps.patches),
                                      "/".join(map(str, planes)), threads, timed,
                                      args.steps, budget_s, iters_per_step)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def profile_batched(ngrids=64):
    """Two steps of a batch of the config-4 generator's first `ngrids` grids
    (FP64, periodic boundaries, the configuration the autotuner picks for the
    full batch: 16x8x32 tiles, two cells per thread), launched directly (no
    graph), for an ncu capture of k_batched_stage and k_batched_ghosts."""
    from lsmlib_b200 import batched, gpu, workloads
    cfg = workloads.config4(ngrids=ngrids)
    b = batched.Batch(cfg["sizes"], cfg["dx"], 8)
    b.upload(workloads.config4_phi(cfg, np.float64))
    b.set_velocity(cfg["vel"], cfg["cfl"])
    b.set_bc(batched.BC_PERIODIC)
    b.set_tile(14)
    b.advect(2, mode=batched.MODE_PERSISTENT)
    gpu.check_rc(gpu.load().lsmgpu_stream_synchronize(), "sync")


def profile_kernels():
    """Two launches each of the normal-velocity and reinitialization stage
    kernels (TVD-RK3 stage 2, distinct phi_s and phi^n, ghost cells read as
    stored: the kernel the drivers launch) on the workload's grid, in FP64
    and then in FP32."""
    from lsmlib_b200 import gpu, integrator, workloads
    cfg = workloads.config2(N_CELLS)
    gb, fb = workloads.boxes(cfg["n"])
    integrator.set_fp_mode(integrator.FP_FAST)
    for prec, dtype in ((8, np.float64), (4, np.float32)):
        a = gpu.DeviceArray(cfg["phi"].shape, dtype)
        b = gpu.DeviceArray.from_host(cfg["phi"].astype(dtype))
        c = gpu.DeviceArray.from_host(cfg["phi"].astype(dtype))
        f = gpu.DeviceArray.from_host(cfg["F"].astype(dtype))
        for kind in (1, 2):
            for _ in range(2):
                integrator.stage(kind, prec, a, b, c, [f], gb, fb, cfg["dx"], 1e-3, 32,
                                 bc_mask=0)
        gpu.check_rc(gpu.load().lsmgpu_stream_synchronize(), "sync")
        del a, b, c, f


def profile_adjoint():
    """The config-5 problem's forward run and reverse sweep, twice (for ncu
    captures of the adjoint stage kernel)."""
    from lsmlib_b200 import adjoint, workloads
    cfg = workloads.config5()
    p = adjoint.AdvectionAdjoint(cfg["n"], cfg["dx"], cfg["x_lo"], cfg["lattice"],
                                 cfg["steps"], 15)
    p.set_theta(cfg["theta"])
    p.set_dt(p.cfl_dt(cfg["cfl"]))
    p.set_fields(cfg["phi0"], cfg["target"], cfg["eps"])
    for _ in range(2):
        p.forward()
        p.backward()
    p.close()


def profile_distance(n=128):
    """The distance function on workloads.distance_case(n), orders 1 and 2,
    device arrays (for ncu captures of the band-solver pass kernel)."""
    from lsmlib_b200 import gpu, workloads
    lib = gpu.load()
    phi, dx = workloads.distance_case(n)
    d_phi = gpu.DeviceArray.from_host(phi)
    d_out = gpu.DeviceArray(phi.shape)
    dims = (ctypes.c_int * 3)(n, n, n)
    h = (ctypes.c_double * 3)(*dx)
    for order in (1, 2):
        gpu.check_rc(lib.lsmgpu_distance_function3d(d_out.ptr, d_phi.ptr, None, order, dims, h,
                                                    None), "distance")
    d_phi.free()
    d_out.free()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity check of the timed configuration")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the CPU baseline sample of our arm")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32 form")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint leg (config 5)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched uneven-grid leg (config 4)")
    ap.add_argument("--no-toolbox", action="store_true",
                    help="skip the per-routine drop-in timings")
    ap.add_argument("--no-distance", action="store_true",
                    help="skip the fast marching leg (distance, extension fields, Eikonal)")
    ap.add_argument("--no-deformation", action="store_true",
                    help="skip the deformation leg (config 3)")
    ap.add_argument("--config3-full", action="store_true",
                    help="run the config-3 full reversal at 512^3 (minutes) instead of 256^3")
    ap.add_argument("--size", type=int, default=256, help="interior cells per axis")
    ap.add_argument("--profile-batched", action="store_true",
                    help="only two steps of a 64-grid batch (for ncu captures) and exit")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="only run the config-5 forward and reverse sweep twice "
                         "(for ncu captures) and exit")
    ap.add_argument("--profile-distance", action="store_true",
                    help="only run the 128^3 distance function at orders 1 and 2 "
                         "(for ncu captures) and exit")
    ap.add_argument("--profile", action="store_true",
                    help="only launch the two fused stage kernels twice each "
                         "(for ncu captures) and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    global N_CELLS
    N_CELLS = args.size
    world, rank, local, pg = dist_setup(args.gpus)
    if args.profile:
        profile_kernels()
        return
    if args.profile_adjoint:
        profile_adjoint()
        return
    if args.profile_batched:
        profile_batched()
        return
    if args.profile_distance:
        profile_distance()
        return
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_ours(args, world, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
