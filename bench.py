#!/usr/bin/env python3
"""Throughput of FVCOM's mode-split time step on B200: cell-layer updates per second.

One "step" is one INTERNAL_STEP (ISPLIT=10 external steps of 4 Runge-Kutta stages, then
the 3-D momentum, turbulence, T/S and density updates) over the whole mesh.  The default
workload is the large coastal mesh: a seeded Delaunay triangulation of 200,000 jittered
points in 200 km x 100 km, 40 sigma layers, wetting/drying on, M2+S2 tide, 10 m/s wind,
plain FP64.  Inputs are synthetic (generated here); no dataset is read.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU runs (torchrun, one rank per GPU) step independent replicas of the mesh: the
single-mesh path does not shard (scaling "weak"); the timed region is bracketed by a
barrier and a device synchronize and the slowest rank's device time is reported.

The reference arm (--impl reference) times the FP64 CPU restatement of the reference
(the oracle: FVCOM's Fortran cannot be built on these machines) on all host cores.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="coastal", choices=["coastal", "channel"])
    ap.add_argument("--npts", type=int, default=200000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shape instead of autotuning it")
    ap.add_argument("--precision", default="fp32flux", choices=["fp64", "fp32flux"],
                    help="form timed for the headline value (fp32flux: FP32 edge fluxes and advection)")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip timing the plain FP64 path beside the chosen form")
    return ap.parse_args()


def make_case(args):
    from myfvcomcode_b200 import cases
    if args.workload == "coastal":
        return cases.coastal_mesh(npts=args.npts, kb=41, seed=1234)
    return cases.estuary_channel()


def workload_config(case, args):
    g, p = case["grid"], case["params"]
    return {
        "workload": case["name"],
        "mesh": "seeded Delaunay of jittered points, 200 km x 100 km" if args.workload == "coastal"
        else "20 km x 4 km channel, 100x20 grid split diagonally",
        "nodes": g["M"], "cells": g["N"], "layers": g["KB"] - 1, "isplit": p["ISPLIT"],
        "dte_s": p["DTE"], "wetting_drying": bool(p["WETTING_DRYING_ON"]),
        "precision": "plain FP64",
        "l2": "inputs larger than L2 (the 3-D fields of one step are several GB)",
        "parallelism": "replicas" if args.gpus > 1 else "single",
    }


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes from the committed ncu summary, if one exists."""
    path = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                try:
                    out[(parts[0], parts[1])] = float(parts[2])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, x, local):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda:%d" % local)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        import torch
        torch.cuda.synchronize(local)
        pg.barrier()


def cpu_rate(case, seconds, warm=1, cap=None):
    """Oracle (FP64 CPU restatement) throughput on all host threads, bounded sample."""
    from oracle.oracle import Oracle, max_threads
    o = Oracle(case)
    o.run(warm)
    t0 = time.perf_counter()
    o.run(1)
    t1 = time.perf_counter() - t0
    n = max(1, int(seconds / max(t1, 1e-9)) - 1)
    if cap:
        n = min(n, cap)
    t0 = time.perf_counter()
    o.run(n)
    dt = time.perf_counter() - t0
    g = case["grid"]
    steps = n + 1
    rate = g["N"] * (g["KB"] - 1) * steps / (dt + t1)
    return rate, max_threads(), steps, dt + t1


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    case = make_case(args)
    g, p = case["grid"], case["params"]
    cells_layers = g["N"] * (g["KB"] - 1)
    cfg = workload_config(case, args)
    metric = "cell-layer updates/s"

    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(1, min(args.steps, 5))
        rate, cores, n, secs = cpu_rate(case, 1e9, warm=min(max(args.warmup, 0), 1), cap=steps - 1)
        line = {"impl": "reference", "metric": metric, "value": rate, "unit": "cell-layer updates/s",
                "n_gpus": args.gpus, "steps": n, "warmup": min(args.warmup, 1),
                "ms_per_step": 1e3 * secs / n, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": rate, "unit": "cell-layer updates/s", "cores": cores, "kind": "port",
                                 "sample": "%d internal steps of the full workload after one warm-up step, "
                                           "FP64 CPU restatement of the reference (OpenMP over layers and "
                                           "columns)" % n},
                "e2e": {"value": rate, "unit": "cell-layer updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import ctypes as C
    from myfvcomcode_b200.engine import Fvcom
    from myfvcomcode_b200 import bytes_model
    if world == 1:
        import torch  # noqa: F401  (pinned host buffers for the end-to-end leg)
    import torch
    torch.cuda.set_device(local)
    lib = None

    def timed_handle(precision):
        """A handle of the case in ``precision``, autotuned and warmed up, and its device
        time over ``args.steps`` internal steps (max over ranks) with the clocks seen."""
        f = Fvcom(case)
        f.set_precision(precision)
        if not args.no_tune:
            from myfvcomcode_b200 import autotune
            tuned = autotune.autotune(case, steps=2, warmup=1, engine=f)
            autotune.apply(f, tuned)
        f.run(args.warmup)
        barrier(pg, local)
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        t = f.time_steps(args.steps)
        clocks = sampler.stop()
        barrier(pg, local)
        t = reduce_max(pg, t, local)
        if f.shutdown_check() != 0:
            raise SystemExit("non-finite state after the timed steps (%s)" % precision)
        return f, t, clocks

    f, t_ms, clocks = timed_handle(args.precision)
    lib = f.lib
    lib.fvg_profile.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.fvg_profile_groups.restype = C.c_int32
    lib.fvg_profile_group_name.restype = C.c_char_p
    lib.fvg_profile_group_name.argtypes = [C.c_int32]
    lib.fvg_kernels_per_step.argtypes = [C.c_void_p]
    lib.fvg_kernels_per_step.restype = C.c_int32
    cfg["precision"] = {"fp64": "plain FP64",
                        "fp32flux": "FP32 edge fluxes/advection/FCT; FP64 elevation update, "
                                    "column solves, state and budgets"}[args.precision]
    cfg["tiling"] = {"col_threads": f.get_tuning("col_threads"), "col_layers": f.get_tuning("col_layers"),
                     "autotuned": not args.no_tune}
    value = cells_layers * args.steps * world / (t_ms / 1e3)

    plain = None
    if args.precision != "fp64" and not args.no_plain:
        fp, tp_ms, _ = timed_handle("fp64")
        plain = {"value": cells_layers * args.steps * world / (tp_ms / 1e3), "ms_per_step": tp_ms / args.steps,
                 "tiling": [fp.get_tuning("col_threads"), fp.get_tuning("col_layers")]}
        # Both handles ran the same steps from the same cold start: live error of the
        # chosen form against FP64 at this point of the run.
        from myfvcomcode_b200.precision_report import compare
        n_done = fp.clock()[0]
        if f.clock()[0] == n_done:
            plain["error_of_chosen_form"] = dict(compare(fp, f), internal_steps=n_done)
        fp.close()
        day = os.path.join(ROOT, "profiles", "precision_error_coastal200k_k40_1day.json")
        if os.path.exists(day):
            with open(day) as fh:
                plain["error_after_1_day"] = json.load(fh).get("errors_vs_fp64")
        cfg["plain_fp64"] = plain

    # per-kernel-group device time (plain launches with events between groups)
    ng = lib.fvg_profile_groups()
    gms = (C.c_double * ng)()
    tot = C.c_double()
    nprof = 2
    lib.fvg_profile(f.h, nprof, gms, C.byref(tot))
    names = [lib.fvg_profile_group_name(i).decode() for i in range(ng)]
    led = bytes_model.ledger(g, p["ISPLIT"], bool(p["WETTING_DRYING_ON"]), args.precision)
    groups = {names[i]: gms[i] / nprof for i in range(ng) if gms[i] > 0}
    dom = max(groups, key=groups.get)
    b_launch, n_launch = led[dom]
    dur = groups[dom] / n_launch
    achieved = b_launch / (dur / 1e3) / 1e9
    peak, peak_kind = peak_hbm()
    traffic = traffic_table().get((dom, case["name"]))
    step_b = bytes_model.step_bytes(g, p["ISPLIT"], bool(p["WETTING_DRYING_ON"]), args.precision)
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": b_launch, "launch_ms": dur,
            "share": groups[dom] / (tot.value / nprof),
            "step_algorithmic_bytes": step_b,
            "step_frac": step_b / (t_ms / args.steps / 1e3) / 1e9 / peak,
            "groups_ms_per_step": {k: round(v, 4) for k, v in sorted(groups.items(), key=lambda kv: -kv[1])}}

    e2e = None
    if not args.no_e2e:
        from myfvcomcode_b200.abi import wind_stress
        ws = wind_stress(case)
        n1 = g["N"] + 1
        hx = torch.zeros(n1, dtype=torch.float64).pin_memory()
        hy = torch.zeros(n1, dtype=torch.float64).pin_memory()
        if ws is not None:
            hx.copy_(torch.from_numpy(ws[0]))
            hy.copy_(torch.from_numpy(ws[1]))
        hel = torch.zeros(g["M"] + 1, dtype=torch.float64).pin_memory()
        dp = C.POINTER(C.c_double)
        lib.fvg_set_field.argtypes = [C.c_void_p, C.c_char_p, dp, C.c_int64]
        lib.fvg_get_field.argtypes = [C.c_void_p, C.c_char_p, dp, C.c_int64]
        px = C.cast(hx.data_ptr(), dp)
        py = C.cast(hy.data_ptr(), dp)
        pe = C.cast(hel.data_ptr(), dp)
        ne = max(3, args.steps // 2)
        barrier(pg, local)
        t0 = time.perf_counter()
        for _ in range(ne):
            lib.fvg_set_field(f.h, b"wstress_x", px, n1)
            lib.fvg_set_field(f.h, b"wstress_y", py, n1)
            lib.fvg_internal_step(f.h)
            lib.fvg_get_field(f.h, b"el", pe, g["M"] + 1)
        te = time.perf_counter() - t0
        te = reduce_max(pg, te, local)
        e2e = {"value": cells_layers * ne * world / te, "unit": "cell-layer updates/s",
               "h2d_bytes_per_step": 2 * n1 * 8, "d2h_bytes_per_step": (g["M"] + 1) * 8,
               "steps": ne, "api": "fvg_set_field(wstress_x/y) + fvg_internal_step + fvg_get_field(el), "
                                   "pinned host buffers, wall clock"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, n, secs = cpu_rate(case, args.cpu_seconds)
        cpu = {"value": rate, "unit": "cell-layer updates/s", "cores": cores, "kind": "port",
               "sample": "%d internal steps (%.1f s) of the full workload after one warm-up step, FP64 "
                         "CPU restatement of the reference on %d threads" % (n, secs, cores)}

    if rank == 0:
        line = {"metric": metric, "value": value, "unit": "cell-layer updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32 fluxes, f64 state",
                "data": "synthetic", "config": cfg, "clocks": clocks, "e2e": e2e, "roofline": roof,
                "cpu_baseline": cpu, "gpu_launches": int(lib.fvg_kernels_per_step(f.h)) * args.steps}
        print(json.dumps(line), flush=True)
    f.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
