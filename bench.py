#!/usr/bin/env python
"""Throughput of the CodeNS hot path on B200: Mcell-iters/s.

One step = one pseudo-time iteration of the Roe-MUSCL / viscous residual and
the matrix-free point-Jacobi implicit update over every block (atsch_num),
graph-captured, on the laminar Navier-Stokes bump channel: 8 blocks of
seeded uneven sizes (48..128 cells per side, ~4M cells), Mach 0.5, Re 1e4,
minmod-limited MUSCL, lmax = 10 Jacobi sweeps, injection / outlet pressure /
adiabatic walls / periodic span and coincident inter-block joins handled on
the device.  The state (~0.2 GB per field) is far larger than L2, so no L2
flush is needed between steps.

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
# algorithmic bytes per real cell (FP64): read W, S(3 faces), vol, write R
# for the residual; read dW, W, S, R, vol and write dW per Jacobi sweep
BYTES_RESIDUAL = 160
BYTES_JACOBI = 240
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
                   help="a 3-block ~0.1M-cell channel (profiling, smoke runs)")
    return p.parse_args()


def make_case(args):
    from codens_b200 import cases
    if args.small:
        case = cases.channel_case([40, 24, 32], 48, 40, seed=2)
    else:
        case = cases.channel_case(seed=2)
    case.scheme.lmax = args.lmax
    return case


def config_of(case, args, n):
    m = case.meta
    return {
        "workload": "laminar NS bump channel, 8 uneven blocks, Roe-MUSCL minmod + viscous, "
                    f"implicit point-Jacobi lmax={args.lmax}, FP64"
        if not args.small else "small laminar NS bump channel (3 blocks)",
        "cells": case.layout.nreal,
        "blocks": case.layout.nblk,
        "block_ni": m.get("ni"), "nj": m.get("nj"), "nk": m.get("nk"),
        "mach": m.get("mach"), "reynolds": m.get("reynz"), "seed": m.get("seed"),
        "precision": "fp64",
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
def cpu_reference_rate(case, steps: int):
    """the oracle (CPU restatement of the reference) on the same case"""
    from oracle.oracle import Oracle, OracleState
    orc = Oracle(case)
    st = OracleState(case)
    orc.metric(st)
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.step(st)
    t = time.perf_counter() - t0
    return case.layout.nreal * steps / t / 1e6, t


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    case = make_case(args)
    # each timed step is a bounded sample: one iteration of the full case
    steps = max(1, min(args.steps, 2))
    for _ in range(min(args.warmup, 0)):
        pass
    rate, t = cpu_reference_rate(case, steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
        "n_gpus": args.gpus, "steps": steps, "warmup": 0,
        "ms_per_step": 1e3 * t / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_of(case, args, 1),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"{steps} iteration(s) of the full case on one core "
                                   "(serial C restatement of the reference; the Fortran "
                                   "reference cannot be built in this image)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if ws > 1:
            dist.barrier()

    from codens_b200.solver import CodeNS

    case = make_case(args)
    s = CodeNS(case, device=local)
    s.metric()
    nreal = case.layout.nreal
    # warm-up (also instantiates the step graph)
    s.atsch_num(max(args.warmup, 3))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    prop = torch.cuda.get_device_properties(local)
    try:
        bus = "%08X:%02X:%02X.0" % (prop.pci_domain_id, prop.pci_bus_id, prop.pci_device_id)
    except Exception:
        bus = None
    sampler = ClockSampler(bus)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0.record(s.stream)
    s.atsch_num_launch(args.steps)
    ev1.record(s.stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    norms = s.last_norms()
    t_max = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms = float(t_max.item())
    value = ws * nreal * args.steps / (ms * 1e-3) / 1e6
    launches_per_step = 15 + args.lmax + (3 if case.scheme.ilim else 0) + (
        1 if any(b.kind == 4 for b in case.boundaries) else 0)

    # dominant-kernel roofline: one Jacobi sweep, timed live on the solver's
    # stream as (implicit phase with lmax sweeps - with 0 sweeps) / lmax
    def time_implicit(lmx, reps=3):
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        for _ in range(reps):
            s.implimf_3d(0, s.u, s.dt, s.v, s.d, s.mu, s.mut, s.sn,
                         s.vol, s.pression, s.cson, lmx)
        b.record(s.stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    def time_residual(reps=3):
        s.sync()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(s.stream)
        for _ in range(reps):
            s.sch_roe(0, s.u, s.v, s.tau, s.sn, s.pression)
        b.record(s.stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    v_keep = s.v.clone()
    t_res = time_residual()
    t_i0 = time_implicit(0)
    t_il = time_implicit(args.lmax)
    s.v.copy_(v_keep)
    torch.cuda.synchronize()
    t_sweep = max((t_il - t_i0) / max(args.lmax, 1), 1e-9)
    hbm, hbm_kind = peaks()
    ach_sweep = BYTES_JACOBI * nreal / (t_sweep * 1e-3) / 1e9
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
    te = time.perf_counter() - t0
    te_t = torch.tensor([te], dtype=torch.float64, device="cuda")
    if ws > 1:
        dist.all_reduce(te_t, op=dist.ReduceOp.MAX)
    te = float(te_t.item())
    e2e = ws * nreal * ne / te / 1e6
    bytes_v = 5 * case.layout.ld * 8

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, tc = cpu_reference_rate(case, args.cpu_steps)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{args.cpu_steps} iteration(s) of the full case, serial C "
                         f"restatement of the reference on one host core ({tc:.1f} s)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_of(case, args, ws),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": bytes_v,
                    "d2h_bytes_per_step": bytes_v + 15 * 8},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "kernel": "Jacobi sweep (k_jacobi)",
                         "achieved": ach_sweep, "peak": hbm, "unit": "GB/s",
                         "frac": ach_sweep / hbm, "peak_source": hbm_kind,
                         "traffic": None, "ms_per_launch": t_sweep,
                         "bytes_per_launch": BYTES_JACOBI * nreal},
            "roofline_residual": {"bound": "hbm", "achieved": ach_res, "peak": hbm,
                                  "unit": "GB/s", "frac": ach_res / hbm,
                                  "ms_per_launch": t_res},
            "clocks": clocks,
            "final_l2_rho": float(norms[1, 0]),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    s.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
