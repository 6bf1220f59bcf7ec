#!/usr/bin/env python
"""Throughput of the CodeNS hot path on B200: Mcell-iters/s.

One step = one pseudo-time iteration of the Roe-MUSCL / viscous residual and
the matrix-free point-Jacobi implicit update over every block (atsch_num),
graph-captured, on the laminar Navier-Stokes bump channel: 8 blocks of
seeded uneven sizes (48..128 cells per side, ~4.4M cells), Mach 0.5, Re 1e4,
kappa = -1 MUSCL, lmax = 10 Jacobi sweeps, injection / outlet pressure /
adiabatic walls / periodic span and coincident inter-block joins handled on
the device.  The state (~0.2 GB per field) is far larger than L2, so no L2
flush is needed between steps.

The headline value is the mixed form (FP64 residual, boundary conditions,
update and norms; FP32 Jacobi sweeps), whose fixed point is the FP64 steady
state; the plain FP64 iteration is timed in the same run beside it, and a
small viscous box is converged in both forms to state the equal-error claim
(`steady_state`).

Arms:
  default            the CUDA path (device-resident state, CUDA events on the
                     solver's stream); e2e through cns_atsch_num_step_host
                     (pinned host state copied in and out every step)
  --impl reference   the CPU restatement of the reference (oracle/) on the
                     host cores, a bounded number of iterations of the same case

Multi-GPU (torchrun): replicas only -- every rank runs its own channel, no
data-path collective; value = all ranks' cell-iterations / the slowest rank.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-iters/s, mixed-prec vs FP64 GPU at equal L2 error; adjoint/primal cost"
UNIT = "Mcell-iters/s"
# algorithmic bytes per real cell: read W, S (3 owned faces), vol, write R
# for the residual (FP64); read dW, W, S, R, vol and write dW per Jacobi
# sweep, at the stored element size (FP64: 240 B, FP32: 120 B)
BYTES_RESIDUAL = 160
BYTES_JACOBI = {"fp64": 240, "mixed": 120, "defect": 120}
PRECISION = {"fp64": 0, "mixed": 1, "defect": 2}
DTYPE = {"fp64": "f64", "mixed": "f64 residual/update, f32 sweeps",
         "defect": "f32 fluxes/sweeps, f64 accumulate/update"}
SWEEP_KERNEL = {"fp64": "k_jacobi_25d<double> (2.5D point-Jacobi sweep, recomputed increments)",
                "mixed": "k_sweep_f32 (persistent 2.5D point-Jacobi sweep, FP32 increments)",
                "defect": "k_sweep_f32 (persistent 2.5D point-Jacobi sweep, FP32 increments)"}
# DRAM bytes per cell of one 2.5D sweep launch, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the 1.18M-cell channel;
# traffic grows with the cells processed, so a full launch is this x cells
SWEEP_TRAFFIC_PER_CELL = {"fp64": 326.4, "mixed": 152.0, "defect": 152.0}
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--lmax", type=int, default=10)
    p.add_argument("--e2e-steps", type=int, default=20)
    p.add_argument("--cpu-steps", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--small", action="store_true",
                   help="a 3-block 1.18M-cell channel (profiling captures)")
    p.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "defect"])
    p.add_argument("--kdefect", type=int, default=4, help="defect form: FP64 refresh period")
    p.add_argument("--no-fp64-arm", action="store_true",
                   help="skip timing the plain FP64 iteration beside the mixed one")
    p.add_argument("--no-steady-check", action="store_true")
    p.add_argument("--no-minmod", action="store_true",
                   help="skip timing the minmod-limited (ilim 1) iteration beside the headline")
    p.add_argument("--no-c1", action="store_true",
                   help="skip the 64x32x32 box sub-runs 1a/1b/1c")
    p.add_argument("--rans-iters", type=int, default=3000,
                   help="rans workload: iterations of the convergence history")
    p.add_argument("--workload", default="channel",
                   choices=["channel", "batch", "adjoint", "rans", "dual"],
                   help="channel: the 8-block NS channel; batch: 64 independent Euler boxes "
                        "in one launch against the same boxes one at a time")
    p.add_argument("--residual-tiles", default=None,
                   help="TI,TJ,KC: the fused residual kernel with these 2.5D tiles (32,4 or "
                        "16,8) instead of the face kernels + accumulation")
    p.add_argument("--tune-cache", default=None,
                   help="sweep-tiling cache file: a tiling found there is used without timing")
    p.add_argument("--tiles", default=None,
                   help="TI,TJ,KC: fix the Jacobi sweep tiling instead of autotuning it")
    p.add_argument("--sweep-staging", type=int, default=0, choices=[0, 1],
                   help="FP32 sweep plane staging: 0 tensor boxes (TMA), 1 cp.async copies")
    p.add_argument("--eta", type=float, default=5.0,
                   help="CFL number of the local time step (AUSM+ needs 2 on the channel)")
    p.add_argument("--flux", default="roe", choices=["roe", "hllc", "rusanov", "ausm", "weno5"],
                   help="flux family of the channel workload (ischema 7, 14, 9, 5, 12; "
                        "WENO5 with its flagged three-candidate fix, the reference form "
                        "reaching no steady state)")
    p.add_argument("--ilim", type=int, default=0,
                   help="0: plain kappa=-1 MUSCL (default: the reference's limiter "
                        "recurrence stalls this channel at L2 ~1e-3); 1: minmod limiter")
    return p.parse_args()


FLUX = {"roe": 7, "hllc": 14, "rusanov": 9, "ausm": 5, "weno5": 12}
FLUX_NAME = {"roe": "Roe", "hllc": "HLLC", "rusanov": "Rusanov", "ausm": "AUSM+",
             "weno5": "WENO5 (three-candidate fix)"}


def make_case(args):
    from codens_b200 import cases
    if args.small:
        case = cases.channel_case([64, 64, 64], 64, 96, seed=2)
    else:
        case = cases.channel_case(seed=2)
    case.scheme.lmax = args.lmax
    case.scheme.ilim = args.ilim
    case.scheme.ischema = FLUX[args.flux]
    case.scheme.weno_fix = int(args.flux == "weno5")
    case.scheme.eta = args.eta
    case.scheme.precision = PRECISION[args.precision]
    case.scheme.kdefect = args.kdefect
    return case


def config_of(case, args, n):
    m = case.meta
    return {
        "workload": f"laminar NS bump channel, 8 uneven blocks, {FLUX_NAME[args.flux]}"
                    f"{'' if args.flux == 'weno5' else '-MUSCL'}"
                    f"{' minmod' if args.ilim else ''} + viscous, "
                    f"implicit point-Jacobi lmax={args.lmax}, {args.precision}"
        if not args.small else "laminar NS bump channel, 3 blocks of 64x64x96 cells",
        "cells": case.layout.nreal,
        "blocks": case.layout.nblk,
        "block_ni": m.get("ni"), "nj": m.get("nj"), "nk": m.get("nk"),
        "mach": m.get("mach"), "reynolds": m.get("reynz"), "seed": m.get("seed"),
        "precision": args.precision,
        "ilim": args.ilim,
        "residual": (f"fused kernel, tiles {args.residual_tiles}" if args.residual_tiles
                     else "face kernels + accumulation"),
        "flux": args.flux,
        "sweep_staging": "cp.async" if args.sweep_staging else "tensor boxes (TMA)",
        "eta": args.eta,
        "l2_flush": "inputs larger than L2 (state and scratch ~GBs)",
        "parallelism": f"replicas x{n}" if n > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while timing"""

    Q = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus = bus_id
        self.proc = None
        self.path = os.path.join("/tmp", f"cns_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                   "-lms", "100"]
            if self.bus:
                cmd += ["-i", self.bus]
            self.proc = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            try:
                sm.append(float(p[2]))
                smax.append(float(p[3]))
            except ValueError:
                continue
            for nm, val in zip(names, p[6:10]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
def cpu_reference_rate(case, steps: int, threads: int = 0):
    """the oracle (CPU restatement of the reference) on the same case; its
    per-block routines run on up to `threads` host threads (0: all cores),
    block-parallel as the reference's MPI ranks are"""
    from oracle.oracle import Oracle, OracleState, lib
    threads = threads or (os.cpu_count() or 1)
    lib().orc_set_threads(threads)
    orc = Oracle(case)
    st = OracleState(case)
    orc.metric(st)
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.step(st)
    t = time.perf_counter() - t0
    return case.layout.nreal * steps / t / 1e6, t, min(threads, case.layout.nblk)


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    case = make_case(args)
    # each timed step is a bounded sample: one iteration of the full case
    steps = max(1, min(args.steps, 2))
    rate, t, cores = cpu_reference_rate(case, steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * t / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_of(case, args, 1),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{steps} iteration(s) of the full case, the C restatement "
                                   f"of the reference with its per-block routines on {cores} "
                                   "threads (one per block at most, as the reference's MPI "
                                   "ranks); the Fortran reference cannot be built in this "
                                   "image"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def _timed_steps(s, torch, steps):
    """CUDA-event time of `steps` graph-launched iterations on the solver's
    stream (ms), with the kernels they launched"""
    s.sync()
    k0 = s.kernels_launched
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(s.stream)
    s.atsch_num_launch(steps)
    b.record(s.stream)
    b.synchronize()
    return a.elapsed_time(b), s.kernels_launched - k0


def _sweep_ms(s, torch, scheme, lmax, steps):
    """one 2.5D Jacobi sweep (every sweep but the first, which is a cheaper
    per-cell kernel or part of the coefficient kernel), timed live on the
    solver's stream as the difference of the fused iteration with lmax
    sweeps and with one, over `steps` iterations each (ms per sweep)"""
    if lmax < 2:
        return float("nan")
    t_l, _ = _timed_steps(s, torch, steps)
    scheme.lmax = 1
    s.set_scheme(scheme)
    s.atsch_num_launch(3)
    t_1, _ = _timed_steps(s, torch, steps)
    scheme.lmax = lmax
    s.set_scheme(scheme)
    s.atsch_num_launch(3)
    return max((t_l - t_1) / steps / (lmax - 1), 1e-9)


def _residual_ms(s, torch, reps=5):
    """the FP64 residual of every block with the case's flux family
    (sch_roe / sch_roe_euler, sch_hllc / sch_hllc_euler, sch_rusanov), ms"""
    s.sync()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    ischema = s.case.scheme.ischema
    a.record(s.stream)
    for _ in range(reps):
        if ischema == 9:
            s.sch_rusanov(0, s.u, s.v, s.tau, s.sn, s.pression)
        elif ischema == 12:
            s.sch_weno5_3d(0, s.u, s.v, s.tau, s.sn, s.pression)
        elif ischema == 5:
            s.sch_ausmp(0, s.u, s.v, s.tau, s.sn, s.pression)
        elif ischema == 14 and s.case.scheme.ns:
            s.sch_hllc(0, s.u, s.v, s.tau, s.sn, s.pression)
        elif ischema == 14:
            s.sch_hllc_euler(0, s.u, s.v, s.sn, s.pression)
        elif s.case.scheme.ns:
            s.sch_roe(0, s.u, s.v, s.tau, s.sn, s.pression)
        else:
            s.sch_roe_euler(0, s.u, s.v, s.sn, s.pression)
    b.record(s.stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def steady_state_check(iters=4500):
    """converge a small duct with a unique steady state (inlet and outlet
    conditions, periodic j and k) in the FP64 and the mixed form; the state
    difference relative to the FP64 state's scale (density and energy by
    their largest magnitude, momentum by the largest momentum magnitude)"""
    import numpy as np
    from codens_b200 import cases
    from codens_b200.solver import CodeNS

    out = {}
    states = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        case = cases.channel_case([6, 8, 5], 6, 4, seed=5, reynz=100.0, ilim=0, bump=0.0,
                                  walls=False)
        case.scheme.precision = prec
        s = CodeNS(case)
        s.metric()
        n = s.atsch_num(iters)
        states[name] = s.v.cpu().numpy().reshape(5, case.layout.ld)[:, case.layout.real_cells()]
        out[f"l2_rho_{name}"] = float(n[1, 0])
        s.close()
    a, r = states["mixed"], states["fp64"]
    mom = float(np.sqrt((r[1:4] ** 2).sum(axis=0)).max())
    scale = np.array([np.abs(r[0]).max(), mom, mom, mom, np.abs(r[4]).max()])[:, None]
    out["err_vs_fp64"] = float((np.abs(a - r) / scale).max())
    out["case"] = "viscous duct, 3 blocks of 6..8x6x4 cells, inlet/outlet, Re 100, seed 5"
    out["iters"] = iters
    return out


def c1_runs(torch, steps=100, warm=3):
    """the 64x32x32-cell box (65,536 cells) as its three reference-path
    sub-runs, FP64 and mixed, `steps` graph-launched iterations each on the
    device (the box's state fits in L2: latency- and launch-bound, not an HBM
    case).  1a and 1b run the flagged implimf_eu fix (qfix_dfez = 1): the
    reference form turns non-finite within a few iterations."""
    from codens_b200 import cases
    from codens_b200.solver import CodeNS

    out = {}
    for sub in cases.C1_SUBRUNS:
        rec = {}
        for name, prec in (("fp64", 0), ("mixed", 1)):
            case = cases.c1_case(sub, qfix_dfez=0 if sub == "1c" else 1)
            case.scheme.precision = prec
            s = CodeNS(case)
            s.metric()
            s.atsch_num(warm)
            s.sync()
            k0 = s.kernels_launched
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(s.stream)
            s.atsch_num_launch(steps)
            b.record(s.stream)
            b.synchronize()
            ms = a.elapsed_time(b)
            n = s.last_norms()
            rec[name] = {"value": case.layout.nreal * steps / (ms * 1e-3) / 1e6,
                         "ms_per_step": ms / steps,
                         "kernels_per_step": (s.kernels_launched - k0) / steps,
                         "l2_rho": float(n[1, 0])}
            s.close()
        rec["qfix_dfez"] = 0 if sub == "1c" else 1
        out[sub] = rec
    return out


def run_ours(args):
    import torch

    from codens_b200.replicas import Replicas

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    barrier = rep.barrier
    max_over_ranks = rep.max

    from codens_b200.solver import CodeNS

    case = make_case(args)
    s = CodeNS(case, device=local)
    s.metric()
    if args.tune_cache:
        s.set_tune_cache(args.tune_cache)
    if args.residual_tiles:
        s.set_residual_tiles(*(int(x) for x in args.residual_tiles.split(",")))
    if args.sweep_staging:
        s.set_sweep_staging(args.sweep_staging)
    if args.tiles:
        ti, tj, kc = (int(x) for x in args.tiles.split(","))
        s.set_sweep_tiles(PRECISION[args.precision], ti, tj, kc)
        if args.precision != "fp64":
            s.set_sweep_tiles(0, ti, tj, kc)
    nreal = case.layout.nreal
    warm = max(args.warmup, 3)
    # warm-up (also instantiates the step graphs)
    s.atsch_num(warm)
    prop = torch.cuda.get_device_properties(local)
    try:
        bus = "%08X:%02X:%02X.0" % (prop.pci_domain_id, prop.pci_bus_id, prop.pci_device_id)
    except Exception:
        bus = None
    sampler = ClockSampler(bus)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ms, kernels = _timed_steps(s, torch, args.steps)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    tiles = s.sweep_tiles(PRECISION[args.precision])
    barrier()
    norms = s.last_norms()
    ms = max_over_ranks(ms)
    value = ws * nreal * args.steps / (ms * 1e-3) / 1e6

    # the plain FP64 iteration on the same solver, same step count
    fp64 = None
    if args.precision != "fp64" and not args.no_fp64_arm:
        sch = case.scheme
        keep = sch.precision
        sch.precision = 0
        s.set_scheme(sch)
        s.atsch_num(warm)
        barrier()
        ms64, _ = _timed_steps(s, torch, args.steps)
        barrier()
        ms64 = max_over_ranks(ms64)
        fp64 = {"value": ws * nreal * args.steps / (ms64 * 1e-3) / 1e6,
                "ms_per_step": ms64 / args.steps}
        sch.precision = keep
        s.set_scheme(sch)
        s.atsch_num(warm)

    # dominant-kernel roofline (the Jacobi sweep of the selected form) and
    # the FP64 residual, timed live on the solver's stream
    hbm, hbm_kind = peaks()
    v_keep = s.v.clone()
    nsw = max(5, min(args.steps, 20))
    t_sweep = _sweep_ms(s, torch, case.scheme, args.lmax, nsw)
    t_res = _residual_ms(s, torch)
    s.v.copy_(v_keep)
    torch.cuda.synchronize()
    # the single-sweep iterations of the sweep timing can leave the state
    # (restored above) on a diverging path, e.g. a non-positive temperature
    # at CFL 5; reading the status word once clears what they set
    from codens_b200 import abi as _abi
    try:
        s.last_norms()
    except _abi.CnsError:
        pass
    bj = BYTES_JACOBI[args.precision]
    ach_sweep = bj * nreal / (t_sweep * 1e-3) / 1e9
    ach_res = BYTES_RESIDUAL * nreal / (t_res * 1e-3) / 1e9

    # end to end through the host-array entry point (pinned host state)
    ne = max(1, args.e2e_steps)
    vh = torch.empty(5 * case.layout.ld, dtype=torch.float64).pin_memory()
    vh.copy_(s.v.cpu())
    s.atsch_num_host(vh, 1)
    barrier()
    t0 = time.perf_counter()
    for _ in range(ne):
        s.atsch_num_host(vh, 1)
    te = max_over_ranks(time.perf_counter() - t0)
    e2e = ws * nreal * ne / te / 1e6
    bytes_v = 5 * case.layout.ld * 8

    steady = None
    if rank == 0 and args.precision == "mixed" and not args.no_steady_check:
        steady = steady_state_check()

    # the minmod limiter (ilim = 1: the reference's in-place ratio recurrence,
    # three line-recurrence launches more per iteration), same form and steps
    minmod = None
    if not args.ilim and not args.no_minmod:
        sch = case.scheme
        sch.ilim = 1
        minmod = {}
        for name, prec in ((args.precision, PRECISION[args.precision]), ("fp64", 0)):
            if name in minmod:
                continue
            keep = sch.precision
            sch.precision = prec
            s.set_scheme(sch)
            s.v.copy_(v_keep)
            s.atsch_num(warm)
            barrier()
            msm, _ = _timed_steps(s, torch, args.steps)
            msm = max_over_ranks(msm)
            minmod[name] = {"value": ws * nreal * args.steps / (msm * 1e-3) / 1e6,
                            "ms_per_step": msm / args.steps}
            sch.precision = keep
        sch.ilim = 0
        s.set_scheme(sch)
        s.v.copy_(v_keep)
        torch.cuda.synchronize()

    c1 = None
    if rank == 0 and not args.no_c1:
        c1 = c1_runs(torch, steps=100, warm=warm)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, tc, cores = cpu_reference_rate(case, args.cpu_steps)
        rate1, tc1, _ = cpu_reference_rate(case, 1, threads=1)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{args.cpu_steps} iteration(s) of the full case, the C "
                         f"restatement of the reference, per-block routines on {cores} host "
                         f"threads ({tc:.1f} s)",
               "single_core": {"value": rate1, "unit": UNIT, "cores": 1,
                               "sample": f"1 iteration of the full case on one thread "
                                         f"({tc1:.1f} s)"},
               "host_cores": os.cpu_count()}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": warm,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[args.precision],
            "data": "synthetic (seeded)",
            "config": dict(config_of(case, args, ws),
                           sweep_tiles={"ti": tiles[0], "tj": tiles[1], "kc": tiles[2],
                                        "source": {0: "set", 1: "timed on the data",
                                                   2: "tuning cache"}[tiles[3]]}),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": bytes_v,
                    "d2h_bytes_per_step": bytes_v + 15 * 8},
            "gpu_launches": kernels,
            "roofline": {"bound": "hbm", "kernel": SWEEP_KERNEL[args.precision],
                         "achieved": ach_sweep, "peak": hbm, "unit": "GB/s",
                         "frac": ach_sweep / hbm, "peak_source": hbm_kind,
                         "traffic": SWEEP_TRAFFIC_PER_CELL[args.precision] * nreal,
                         "traffic_source": "ncu DRAM bytes per cell on the 1.18M-cell channel "
                                           "x cells", "ms_per_launch": t_sweep,
                         "bytes_per_launch": bj * nreal, "bytes_per_cell": bj},
            "roofline_residual": {"bound": "hbm", "kernels": "FP64 residual (all blocks)",
                                  "achieved": ach_res, "peak": hbm, "unit": "GB/s",
                                  "frac": ach_res / hbm, "ms_per_launch": t_res,
                                  "bytes_per_cell": BYTES_RESIDUAL},
            "clocks": clocks,
            "final_l2_rho": float(norms[1, 0]),
        }
        if fp64:
            line["fp64"] = fp64
            line["mixed_over_fp64"] = value / fp64["value"]
        if minmod:
            line["minmod_ilim1"] = minmod
        if c1:
            line["c1_box_64x32x32"] = c1
        if steady:
            line["steady_state"] = steady
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    s.close()
    rep.close()
    return 0


def run_batch(args):
    """64 independent Euler boxes (sides 16..96, Mach 0.3..2, angle -5..5 deg,
    1% noise) stepped in one graph-launched iteration, against the same boxes
    run one at a time (one context each) in FP64"""
    import torch
    from codens_b200 import cases
    from codens_b200.solver import CodeNS

    torch.cuda.set_device(0)
    # the flagged fix of implimf_eu.f90:312 keeps the Euler implicit phase
    # finite over the timed iterations (the reference form diverges)
    bt = cases.batch_case(ncase=64, side=(16, 96), seed=4, qfix_dfez=1, lmax=args.lmax)
    nreal = bt.layout.nreal
    warm = max(args.warmup, 3)
    steps = args.steps

    def timed(s, k):
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        s.atsch_num_launch(k)
        e.record(s.stream)
        e.synchronize()
        return a.elapsed_time(e)

    out = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        bt.scheme.precision = prec
        s = CodeNS(bt)
        s.metric()
        s.atsch_num(warm)
        ms = timed(s, steps)
        out[name] = {"value": nreal * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
                     "kernels_per_step": None}
        s.close()
    def one_at_a_time(prec):
        # every box in its own context, all on one stream so that the boxes
        # run one after the other, each its own graph-launched iteration
        members = [cases.batch_member(bt, ib) for ib in range(bt.layout.nblk)]
        one_stream = torch.cuda.Stream()
        solvers = []
        for m in members:
            m.scheme.precision = prec
            sm = CodeNS(m, stream=one_stream)
            sm.metric()
            sm.atsch_num(warm)
            solvers.append(sm)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(one_stream)
        for _ in range(steps):
            for sm in solvers:
                sm.atsch_num_launch(1)
        t1.record(one_stream)
        t1.synchronize()
        ms1 = t0.elapsed_time(t1)
        for sm in solvers:
            sm.close()
        return {"value": nreal * steps / (ms1 * 1e-3) / 1e6, "ms_per_step": ms1 / steps}

    one = one_at_a_time(0)
    one_mixed = one_at_a_time(1)
    line = {
        "metric": METRIC, "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": steps, "warmup": warm, "ms_per_step": out["mixed"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE["mixed"], "data": "synthetic (seeded)",
        "config": {"workload": "batched Euler: 64 independent boxes, sides 16..96, "
                               "Mach 0.3..2.0, angle -5..5 deg, 1% noise, lmax="
                               f"{args.lmax}, one graph-launched iteration for all",
                   "cells": nreal, "cases": bt.layout.nblk, "seed": 4,
                   "qfix_dfez": 1,
                   "l2_flush": "inputs larger than L2 (~17M cells)"},
        "batched_fp64": out["fp64"], "batched_mixed": out["mixed"],
        "one_at_a_time_fp64": one,
        "one_at_a_time_mixed": one_mixed,
        "batched_over_one_at_a_time": out["fp64"]["value"] / one["value"],
        "batched_over_one_at_a_time_mixed": out["mixed"]["value"] / one_mixed["value"],
        "mixed_batched_over_one_at_a_time_fp64": out["mixed"]["value"] / one["value"],
    }
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args):
    """adjoint / primal cost of the wall-force gradient (configuration 5
    form), in the FP64 and the mixed form (FP32 primal sweeps and FP32
    transposed sweeps; FP64 residual and A^T lambda): per-iteration cost at
    512x256x4 cells, and the converged totals (primal to L2 < 1e-12, adjoint
    to a 1e-10 relative residual) on a 128x64x4 channel, where the full size
    would not converge within a bench run"""
    import torch
    from codens_b200 import adjoint
    from codens_b200.solver import CodeNS

    torch.cuda.set_device(0)
    warm = max(args.warmup, 3)
    k = max(args.steps, 20)
    forms = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        d5 = adjoint.Design(ni=512, nj=256, nk=4, precision=prec)
        case = d5.case()
        nreal = case.layout.nreal
        s = CodeNS(case)
        s.metric()
        s.atsch_num(warm)
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        s.atsch_num_launch(k)
        e.record(s.stream)
        e.synchronize()
        ms_primal = a.elapsed_time(e) / k
        s.close()
        g = adjoint.WallForceGradient(d5, d5.mach, d5.alpha, d5.wall(), tol=1e30, max_iter=200,
                                      adj_tol=0.0, adj_max=warm, check=10 ** 9)
        t0 = time.perf_counter()
        g.s.adjoint_prepare()
        g.s.sync()
        t_prep = time.perf_counter() - t0
        _, gW, _, _ = g.value_and_partials()
        g.solve_adjoint(gW)

        def adjoint_ms(n):
            # one solve of n iterations: set-up, an eager first iteration and
            # the graph capture, then n - 1 replays
            g.adj_max = n
            torch.cuda.synchronize()
            a.record(g.s.stream)
            g.solve_adjoint(gW)
            e.record(g.s.stream)
            e.synchronize()
            return a.elapsed_time(e)
        # the per-iteration cost without the solve's fixed set-up: the
        # difference of a 3k- and a k-iteration solve over 2k iterations
        ms_adj = (adjoint_ms(3 * k) - adjoint_ms(k)) / (2 * k)
        g.close()
        # converged totals on a reduced channel
        dr = adjoint.Design(ni=128, nj=64, nk=4, precision=prec)
        t0 = time.perf_counter()
        gr = adjoint.WallForceGradient(dr, dr.mach, dr.alpha, dr.wall(), tol=1e-12,
                                       max_iter=400000, adj_tol=1e-10, adj_max=400000,
                                       check=500)
        torch.cuda.synchronize()
        t_primal = time.perf_counter() - t0
        t0 = time.perf_counter()
        J, gm, ga, gw = gr.gradient()
        torch.cuda.synchronize()
        t_adjoint = time.perf_counter() - t0
        conv = {"cells": gr.case.layout.nreal, "primal_iters": gr.iters, "primal_l2": gr.l2,
                "primal_s": t_primal, "adjoint_iters": gr.adj_iters,
                "adjoint_residual": gr.adj_hist[-1] if gr.adj_hist else None,
                "adjoint_s": t_adjoint, "adjoint_over_primal": t_adjoint / t_primal,
                "J": J, "dJ_dmach": gm, "dJ_dalpha_deg": ga}
        gr.close()
        forms[name] = {"cells": nreal, "primal_ms_per_iter": ms_primal,
                       "adjoint_ms_per_iter": ms_adj,
                       "adjoint_over_primal_per_iter": ms_adj / ms_primal,
                       "adjoint_prepare_s": t_prep, "converged_128x64x4": conv}
    f64, mx = forms["fp64"], forms["mixed"]
    line = {
        "metric": METRIC, "value": f64["cells"] / (f64["adjoint_ms_per_iter"] * 1e-3) / 1e6,
        "unit": UNIT, "n_gpus": 1,
        "steps": k, "warmup": warm, "ms_per_step": f64["adjoint_ms_per_iter"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "adjoint of the wall pressure force, Euler bump channel "
                               "512x256x4 cells (first-order Roe), one adjoint iteration "
                               "= A^T lambda + lmax transposed sweeps",
                   "cells": f64["cells"], "lmax": adjoint.Design().lmax},
        "primal_ms_per_iter": f64["primal_ms_per_iter"],
        "adjoint_ms_per_iter": f64["adjoint_ms_per_iter"],
        "adjoint_over_primal_per_iter": f64["adjoint_over_primal_per_iter"],
        "adjoint_prepare_s": f64["adjoint_prepare_s"],
        "converged_128x64x4": f64["converged_128x64x4"],
        "mixed": mx,
        "mixed_gradient_vs_fp64": {
            "dJ_dmach_rel": abs(mx["converged_128x64x4"]["dJ_dmach"] -
                                f64["converged_128x64x4"]["dJ_dmach"]) /
                            abs(f64["converged_128x64x4"]["dJ_dmach"])},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_rans(args):
    """RANS Spalart-Allmaras flat plate (configuration 3 form): one block of
    256x128x64 cells, wall spacing 1e-5 growing by 1.1, Mach 0.3, Re 1e6,
    freestream nu~ = 3 nu, the SA transport step (met_num) in every fused
    iteration; wall distance once in FP64 on the device.  Mixed (headline)
    and FP64 iterations are timed; the mixed run then continues for
    --rans-iters iterations to report the residual drop."""
    import torch
    from codens_b200 import cases
    from codens_b200.solver import CodeNS

    torch.cuda.set_device(0)
    warm = max(args.warmup, 3)
    steps = args.steps

    def timed(s, k):
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        s.atsch_num_launch(k)
        e.record(s.stream)
        e.synchronize()
        return a.elapsed_time(e)

    out = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        case = cases.flat_plate_case(lmax=args.lmax)
        case.scheme.precision = prec
        nreal = case.layout.nreal
        s = CodeNS(case)
        s.metric()
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        dist = s.atcaldis3()
        e.record(s.stream)
        e.synchronize()
        ms_dist = a.elapsed_time(e)
        # the flagged source fix: the reference's S~ reaches zero in the
        # freestream of this plate within ~80 iterations (cfke inf / NaN)
        s.set_sa(dist, case.meta["rokinf"], 0.0, 1e-8, stilde_fix=1)
        first = s.atsch_num(1)[1, 0]
        s.atsch_num(warm - 1)
        ms = timed(s, steps)
        # the transport step alone (met_num on the bound state)
        s.sync()
        a.record(s.stream)
        for _ in range(5):
            s.met_num()
        e.record(s.stream)
        e.synchronize()
        ms_sa = a.elapsed_time(e) / 5
        rec = {"value": nreal * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
               "sa_step_ms": ms_sa, "wall_distance_ms": ms_dist,
               "kernels_launched": s.kernels_launched}
        if name == "mixed":
            hist = []
            n = args.rans_iters
            chunk = max(1, n // 10)
            done = 0
            while done < n:
                k = min(chunk, n - done)
                hist.append((warm + steps + 5 + done + k, float(s.atsch_num(k)[1, 0])))
                done += k
            rec["l2_rho_first"] = float(first)
            rec["l2_rho_history"] = hist
            rec["l2_drop"] = hist[-1][1] / float(first) if hist else None
            v = s.v.view(7, -1)
            rc = torch.as_tensor(case.layout.real_cells(), device=s.dev)
            rec["mut_over_mu_max"] = float((s.mut[rc] / s.mu[rc]).max())
            rec["finite"] = bool(torch.isfinite(v).all())
        out[name] = rec
        s.close()
    line = {
        "metric": METRIC, "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": steps, "warmup": warm, "ms_per_step": out["mixed"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE["mixed"], "data": "synthetic (uniform freestream start)",
        "config": {"workload": "RANS Spalart-Allmaras flat plate, one block 256x128x64, "
                               "wall spacing 1e-5 ratio 1.1, Mach 0.3, Re 1e6, nu~ = 3 nu, "
                               f"Roe-MUSCL + viscous, lmax={args.lmax}, met_num every "
                               "iteration",
                   "cells": nreal, "eta": case.scheme.eta,
                   "sa_source": "modified vorticity (Allmaras, Johnson & Spalart 2012), "
                                "non-reference flag stilde_fix=1",
                   "l2_flush": "inputs larger than L2 (~2 GB of state and scratch)"},
        "fp64": out["fp64"], "mixed": out["mixed"],
        "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
    }
    print(json.dumps(line), flush=True)
    return 0


def run_dual(args):
    """Dual time stepping (kfmg = 3) on the channel workload: the fused
    pseudo-time iteration with sch_dual and the physical time term, FP64 and
    mixed, against the steady iteration of the same case; the physical-step
    update (sch_duup) and sch_dual alone; and one physical step run to an
    inner tolerance through the host loop (a norm read per iteration)."""
    import torch
    from codens_b200.solver import CodeNS

    torch.cuda.set_device(0)
    warm = max(args.warmup, 3)
    steps = args.steps
    dt_phys = 0.05

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(s, k):
        s.sync()
        a, e = ev(), ev()
        a.record(s.stream)
        s.atsch_num_launch(k)
        e.record(s.stream)
        e.synchronize()
        return a.elapsed_time(e)

    out = {}
    for name in ("fp64", "mixed"):
        case = make_case(args)
        case.scheme.precision = PRECISION[name]
        case.scheme.kfmg, case.scheme.dt1min = 3, dt_phys
        nreal = case.layout.nreal
        s = CodeNS(case)
        s.metric()
        s.sch_duin()
        s.set_dual_cycle(2)          # the BDF2 form of every later physical step
        s.atsch_num(warm)
        ms = timed(s, steps)
        s.sync()
        a, e = ev(), ev()
        a.record(s.stream)
        for _ in range(5):
            s.sch_duup()
        e.record(s.stream)
        e.synchronize()
        ms_duup = a.elapsed_time(e) / 5
        a.record(s.stream)
        for _ in range(5):
            for l in range(1, case.layout.nblk + 1):
                s.sch_dual(l, s.u, s.v, 2, s.vol, s.ptdual)
        e.record(s.stream)
        e.synchronize()
        ms_dual = a.elapsed_time(e) / 5
        rec = {"value": nreal * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
               "sch_duup_ms": ms_duup, "sch_dual_ms": ms_dual,
               "kernels_launched": s.kernels_launched}
        # one physical step to an inner tolerance of 1e-2 through the host loop
        s.sync()
        t0 = time.perf_counter()
        counts = s.dual_time(1, 200, 1e-2, start=True)
        s.sync()
        rec["physical_step"] = {"inner_iterations": counts[0],
                                "wall_ms": (time.perf_counter() - t0) * 1e3}
        s.close()
        # the steady iteration of the same case, for the cost of the dual terms
        case.scheme.kfmg = 0
        s = CodeNS(case)
        s.metric()
        s.atsch_num(warm)
        ms0 = timed(s, steps)
        rec["steady_ms_per_step"] = ms0 / steps
        rec["dual_over_steady_time"] = (ms / steps) / (ms0 / steps)
        s.close()
        out[name] = rec
    line = {
        "metric": METRIC, "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": steps, "warmup": warm, "ms_per_step": out["mixed"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPE["mixed"], "data": "synthetic (seeded noisy freestream)",
        "config": {**config_of(case, args, 1),
                   "workload": "dual time stepping (kfmg 3, BDF2) on the laminar NS bump "
                               f"channel, physical step {dt_phys}, lmax={args.lmax}",
                   "dt1min": dt_phys},
        "fp64": out["fp64"], "mixed": out["mixed"],
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "rans":
        return run_rans(args)
    if args.workload == "dual":
        return run_dual(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
