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
    ap.add_argument("--workload", default="coastal", choices=["coastal", "channel", "ensemble"])
    ap.add_argument("--members-small", type=int, default=32,
                    help="ensemble: members on the 50k-node 30-layer mesh (all ranks together)")
    ap.add_argument("--members-large", type=int, default=8,
                    help="ensemble: members on the 200k-node 40-layer mesh (all ranks together)")
    ap.add_argument("--closure", default=None,
                    help="a trained closure (.npz from myfvcomcode_b200.closure) for the learned form")
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
    ap.add_argument("--no-combined", action="store_true",
                    help="skip the combined form (FP32 fluxes + learned closure + batched members)")
    ap.add_argument("--combined-large", type=int, default=2,
                    help="combined form: members on the 200k-node 40-layer mesh")
    ap.add_argument("--combined-small", type=int, default=8,
                    help="combined form: members on the 50k-node 30-layer mesh")
    ap.add_argument("--combined-spinup", type=int, default=240,
                    help="combined form: internal steps from the cold start before timing, so that the "
                         "learned closure's columns have left the cold start's state (outside its envelope)")
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
    from myfvcomcode_b200 import dist
    d = dist.setup()
    return d.world, d.rank, d.local, (d if d.pg is not None else None)


def reduce_max(pg, x, local):
    return x if pg is None else pg.reduce_max(x)


def barrier(pg, local):
    if pg is not None:
        pg.barrier()


def cpu_rate(case, seconds, warm=1, cap=None, keep=False):
    """Oracle (FP64 CPU restatement) throughput on all host threads, bounded sample.
    With ``keep`` the stepped oracle is returned too (for the parity check)."""
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
    if keep:
        return rate, max_threads(), steps, dt + t1, o
    o.close()
    return rate, max_threads(), steps, dt + t1


def cpu_rate_single_core(case):
    """One internal step of the oracle on one host thread (after one warm-up step)."""
    from oracle.oracle import Oracle, max_threads, set_threads
    nt = max_threads()
    set_threads(1)
    try:
        o = Oracle(case)
        o.run(1)
        t0 = time.perf_counter()
        o.run(1)
        dt = time.perf_counter() - t0
        o.close()
    finally:
        set_threads(nt)
    g = case["grid"]
    return g["N"] * (g["KB"] - 1) / dt, dt


PARITY_FIELDS = ("el", "ua", "va", "u", "v", "w", "t1", "s1", "q2", "q2l", "km", "kh")


def parity_vs_oracle(case, ora, steps):
    """The plain FP64 library stepped ``steps`` internal steps from the same cold start as
    the oracle ``ora``: per field the max-normalised difference max|a-b|/max|b|, the
    largest per-element relative difference |a-b|/max(|b|, 1e-6 max|b|), and whether the
    two are bitwise equal; the wet/dry flags compared exactly."""
    import numpy as np
    from myfvcomcode_b200.engine import Fvcom
    gpu = Fvcom(case)
    gpu.run(steps)
    g = case["grid"]
    node_fields = ("el", "t1", "s1", "q2", "q2l", "km", "kh")
    out, bitwise = {}, True
    for n in PARITY_FIELDS:
        a, b = gpu.get(n), ora.get(n)
        L = g["M"] + 1 if n in node_fields else g["N"] + 1
        a = a.reshape((L, -1), order="F")[1:]
        b = b.reshape((L, -1), order="F")[1:]
        d = np.abs(a - b)
        scale = float(np.abs(b).max())
        floor = max(1e-6 * scale, 1e-300)
        eq = bool(np.array_equal(a, b))
        bitwise = bitwise and eq
        out[n] = {"max_norm": float(d.max()) / max(scale, 1e-300),
                  "per_element": float((d / np.maximum(np.abs(b), floor)).max()), "bitwise": eq}
    wet = all(np.array_equal(gpu.get(n), ora.get(n)) for n in ("iswetn", "iswetc"))
    same_clock = gpu.clock() == ora.clock()
    gpu.close()
    worst = max(v["max_norm"] for v in out.values())
    return {"steps": steps, "against": "oracle (FP64 CPU restatement), same cold start",
            "form": "plain FP64", "max_rel": worst, "bitwise": bitwise, "wet_dry_flags_equal": wet,
            "clock_equal": same_clock, "fields": out}


def run_ensemble(args, world, rank, local, pg):
    """Batched ensemble: perturbed members of two meshes, each mesh's members as one union
    model, both models stepped by one CUDA graph per internal step.  Members are sharded
    over the ranks (no data-path collective)."""
    import torch
    from myfvcomcode_b200 import autotune, cases, ensemble
    from myfvcomcode_b200.engine import Fvcom, Group
    from myfvcomcode_b200.precision_report import compare
    torch.cuda.set_device(local)
    groups = [("50k-k30", cases.coastal_mesh(npts=50000, kb=31), args.members_small, 5),
              ("200k-k40", cases.coastal_mesh(npts=args.npts, kb=41), args.members_large, 6)]
    trained = None
    if args.closure:
        from myfvcomcode_b200 import closure
        trained = closure.load(args.closure)
    models, unions, cfg_members, bases = [], [], [], []
    cells_layers = 0
    for name, base, n, seed in groups:
        specs = ensemble.perturbed_members(base, n, seed=seed)
        from myfvcomcode_b200.dist import shard
        mine = shard(specs, rank, world)
        if not mine:
            continue
        u = ensemble.union_case(base, mine)
        f = Fvcom(u)
        f.set_precision(args.precision)
        if trained is not None:
            closure.attach(f, trained)
        t = autotune.autotune(u, steps=2, warmup=1, engine=f)
        autotune.apply(f, t)
        models.append(f)
        unions.append((u, mine, base))
        cells_layers += u["grid"]["N"] * (u["grid"]["KB"] - 1)
        cfg_members.append({"mesh": name, "members_this_rank": len(mine), "members_total": n,
                            "tiling": [t["col_threads"], t["col_layers"]]})
    grp = Group(models)
    grp.run(args.warmup)
    barrier(pg, local)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    t_ms = grp.time_steps(args.steps)
    clocks = sampler.stop()
    barrier(pg, local)
    t_ms = reduce_max(pg, t_ms, local)
    total_cl = cells_layers * world  # every rank holds the same member count up to rounding
    value = total_cl * args.steps / (t_ms / 1e3)
    # per-member error of member 0 of each model against its standalone FP64 run
    errors = []
    if rank == 0:
        for f, (u, mine, base) in zip(models, unions):
            n_done = f.clock()[0]
            ref = Fvcom(ensemble.member_case(base, mine[0]))
            ref.run(n_done)

            class _Member:
                KB = f.KB

                def get(self, nm):
                    return ensemble.member_slice(u, 0, nm, f)

                def get3(self, nm):
                    a = self.get(nm)
                    return a.reshape((a.size // self.KB, self.KB), order="F")
            err = compare(ref, _Member())
            errors.append({"mesh": u["name"], "internal_steps": n_done, "errors_vs_fp64_member": err})
            ref.close()
    import ctypes as C
    kps = 0
    for f in models:
        f.lib.fvg_kernels_per_step.argtypes = [C.c_void_p]
        f.lib.fvg_kernels_per_step.restype = C.c_int32
        kps += int(f.lib.fvg_kernels_per_step(f.h))
    grp.close()
    for f in models:
        f.close()
    if rank == 0:
        line = {"metric": "cell-layer updates/s", "value": value, "unit": "cell-layer updates/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32 fluxes, f64 state", "data": "synthetic",
                "config": {"workload": "ensemble", "members": cfg_members, "precision": args.precision,
                           "learned_closure": bool(trained is not None),
                           "launch": "one CUDA graph per internal step holding every model",
                           "perturbations": "wind x U(0.8,1.2), tide amplitude x U(0.9,1.1), T0 + N(0,0.5)"},
                "clocks": clocks, "member_errors": errors,
                "gpu_launches": kps * args.steps}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.close()


def e2e_leg(f, case, args, pg, local, world):
    """The metric end to end through the public C ABI with host buffers: per step the wind
    stress is copied in from pinned host memory, fvg_internal_step runs, and the surface
    elevation is read back; wall clock, max over ranks."""
    import ctypes as C
    import torch
    from myfvcomcode_b200.abi import wind_stress
    g = case["grid"]
    lib = f.lib
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
        rc = lib.fvg_set_field(f.h, b"wstress_x", px, n1)
        rc |= lib.fvg_set_field(f.h, b"wstress_y", py, n1)
        rc |= lib.fvg_internal_step(f.h)
        rc |= lib.fvg_get_field(f.h, b"el", pe, g["M"] + 1)
        if rc:
            raise SystemExit("end-to-end leg: a C-ABI call failed")
    te = time.perf_counter() - t0
    te = reduce_max(pg, te, local)
    return {"value": g["N"] * (g["KB"] - 1) * ne * world / te, "unit": "cell-layer updates/s",
            "h2d_bytes_per_step": 2 * n1 * 8, "d2h_bytes_per_step": (g["M"] + 1) * 8,
            "steps": ne, "api": "fvg_set_field(wstress_x/y) + fvg_internal_step + fvg_get_field(el), "
                                "pinned host buffers, wall clock"}


def combined_leg(args, case, plain_value, local):
    """The chosen form of all three together, on one GPU: FP32 edge fluxes and advection,
    the learned closure (the network trained on the 50k-node coastal mesh, MY2.5 as the
    per-column fallback), and batching: perturbed members of the 200k-node 40-layer mesh
    and of a 50k-node 30-layer mesh, each mesh's members as one union model, both models
    stepped by one CUDA graph per internal step.  Member counts are a reduced ensemble
    (``--combined-large`` and ``--combined-small``; the full 64 + 16 configuration is
    ``--workload ensemble`` over several GPUs).  Returns the throughput over all members,
    its ratio to the plain FP64 single-model rate, and member 0 of each mesh against its
    own plain FP64 run after the same steps."""
    from myfvcomcode_b200 import cases, closure, ensemble
    from myfvcomcode_b200.engine import Fvcom, Group
    from myfvcomcode_b200.precision_report import compare
    trained = closure.load(os.path.join(ROOT, "myfvcomcode_b200", "data", "closure_coastal50k_8seeds.npz"))
    bases = [("200k-k40", case, args.combined_large, 6),
             ("50k-k30", cases.coastal_mesh(npts=50000, kb=31, seed=1234), args.combined_small, 5)]
    models, unions, members = [], [], []
    cells_layers = 0
    for name, base, n, seed in bases:
        if n <= 0:
            continue
        specs = ensemble.perturbed_members(base, n, seed=seed)
        u = ensemble.union_case(base, specs)
        f = Fvcom(u)
        f.set_precision("fp32flux")
        closure.attach(f, trained)
        models.append(f)
        unions.append((u, specs, base))
        cells_layers += u["grid"]["N"] * (u["grid"]["KB"] - 1)
        members.append({"mesh": name, "members": n})
    grp = Group(models)
    grp.run(max(args.warmup, args.combined_spinup))
    t_ms = grp.time_steps(args.steps)
    value = cells_layers * args.steps / (t_ms / 1e3)
    errors = []
    for f, (u, specs, base) in zip(models, unions):
        n_done = f.clock()[0]
        ref = Fvcom(ensemble.member_case(base, specs[0]))
        ref.run(n_done)

        class _Member:
            KB = f.KB

            def get(self, nm):
                return ensemble.member_slice(u, 0, nm, f)

            def get3(self, nm):
                a = self.get(nm)
                return a.reshape((a.size // self.KB, self.KB), order="F")
        errors.append({"mesh": u["name"], "internal_steps": n_done,
                       "columns_on_network": closure.status(f)["columns_on_network"],
                       "member0_vs_plain_fp64": compare(ref, _Member())})
        ref.close()
    import ctypes as C
    kps = 0
    for f in models:
        f.lib.fvg_kernels_per_step.argtypes = [C.c_void_p]
        f.lib.fvg_kernels_per_step.restype = C.c_int32
        kps += int(f.lib.fvg_kernels_per_step(f.h))
    grp.close()
    for f in models:
        f.close()
    return {"value": value, "unit": "cell-layer updates/s", "ms_per_step": t_ms / args.steps,
            "vs_plain_fp64": value / plain_value if plain_value else None,
            "form": "FP32 fluxes + learned closure (BF16 tensor cores, MY2.5 fallback) + batched members, "
                    "one CUDA graph per internal step",
            "members": members, "errors": errors, "gpu_launches": kps * args.steps,
            "timing": "CUDA events around %d group steps after %d steps from the cold start"
                      % (args.steps, max(args.warmup, args.combined_spinup))}


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    if args.workload == "ensemble" and args.impl != "reference":
        run_ensemble(args, world, rank, local, pg)
        return
    case = make_case(args)
    g, p = case["grid"], case["params"]
    cells_layers = g["N"] * (g["KB"] - 1)
    cfg = workload_config(case, args)
    metric = "cell-layer updates/s"

    if args.impl == "reference":
        if rank != 0:
            return
        # the requested warm-up and timed steps, each one internal step of the full workload
        # (about 3 s on 16 host threads); at most 60 timed steps keep the arm within minutes
        from oracle.oracle import Oracle, max_threads
        steps = max(1, min(args.steps, 60))
        warm = max(0, min(args.warmup, 10))
        ora = Oracle(case)
        ora.run(warm)
        t0 = time.perf_counter()
        ora.run(steps)
        secs = time.perf_counter() - t0
        ora.close()
        n, cores = steps, max_threads()
        rate = cells_layers * n / secs
        rate1, secs1 = cpu_rate_single_core(case)
        line = {"impl": "reference", "metric": metric, "value": rate, "unit": "cell-layer updates/s",
                "n_gpus": args.gpus, "steps": n, "warmup": warm,
                "ms_per_step": 1e3 * secs / n, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": rate, "unit": "cell-layer updates/s", "cores": cores, "kind": "port",
                                 "sample": "%d internal steps of the full workload after %d warm-up steps, "
                                           "FP64 CPU restatement of the reference (OpenMP over layers and "
                                           "columns)" % (n, warm),
                                 "single_core": {"value": rate1, "unit": "cell-layer updates/s", "cores": 1,
                                                 "sample": "1 internal step (%.1f s) after one warm-up "
                                                           "step, one host thread" % secs1}},
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
    cfg["compact_stage_kernel"] = bool(f.get_tuning("compact"))
    cfg["tiling"] = {"col_threads": f.get_tuning("col_threads"), "col_layers": f.get_tuning("col_layers"),
                     "autotuned": not args.no_tune}
    value = cells_layers * args.steps * world / (t_ms / 1e3)

    plain = None
    fp = None
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
        # The one-day error report is embedded only when it was made from the library
        # sources and case generator this run is built from (its recorded stamp).
        from myfvcomcode_b200.precision_report import sources_stamp
        day = os.path.join(ROOT, "myfvcomcode_b200", "data", "precision_error_coastal200k_k40_1day.json")
        if os.path.exists(day):
            with open(day) as fh:
                rep = json.load(fh)
            stamp = sources_stamp()
            if rep.get("sources_sha256") == stamp:
                plain["error_after_1_day"] = {"errors_vs_fp64": rep.get("errors_vs_fp64"),
                                              "budget_drift": rep.get("budget_drift"),
                                              "sources_sha256": stamp, "made_at_commit": rep.get("commit")}
            else:
                plain["error_after_1_day"] = {"stale": "report made from other sources (%s), this build %s"
                                              % (str(rep.get("sources_sha256"))[:12], stamp[:12])}
        cfg["plain_fp64"] = plain

    # per-kernel-group device time (plain launches with events between groups)
    ng = lib.fvg_profile_groups()
    gms = (C.c_double * ng)()
    tot = C.c_double()
    nprof = 2
    lib.fvg_profile(f.h, nprof, gms, C.byref(tot))
    names = [lib.fvg_profile_group_name(i).decode() for i in range(ng)]
    compact = bool(f.get_tuning("compact"))
    led = bytes_model.ledger(g, p["ISPLIT"], bool(p["WETTING_DRYING_ON"]), args.precision, compact)
    groups = {names[i]: gms[i] / nprof for i in range(ng) if gms[i] > 0}
    dom = max(groups, key=groups.get)
    b_launch, n_launch = led[dom]
    dur = groups[dom] / n_launch
    achieved = b_launch / (dur / 1e3) / 1e9
    peak, peak_kind = peak_hbm()
    traffic = traffic_table().get((dom, case["name"]))
    step_b = bytes_model.step_bytes(g, p["ISPLIT"], bool(p["WETTING_DRYING_ON"]), args.precision, compact)
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": b_launch, "launch_ms": dur,
            "share": groups[dom] / (tot.value / nprof),
            "step_algorithmic_bytes": step_b,
            "step_frac": step_b / (t_ms / args.steps / 1e3) / 1e9 / peak,
            "groups_ms_per_step": {k: round(v, 4) for k, v in sorted(groups.items(), key=lambda kv: -kv[1])}}

    e2e = None
    if not args.no_e2e:
        e2e = e2e_leg(f, case, args, pg, local, world)
    if plain is not None and fp is not None:
        if not args.no_e2e:
            plain["e2e"] = e2e_leg(fp, case, args, pg, local, world)
        fp.close()

    combined = None
    if world == 1 and args.workload == "coastal" and not args.no_combined:
        combined = combined_leg(args, case, plain["value"] if plain else None, local)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, n, secs, ora = cpu_rate(case, args.cpu_seconds, keep=True)
        cpu = {"value": rate, "unit": "cell-layer updates/s", "cores": cores, "kind": "port",
               "sample": "%d internal steps (%.1f s) of the full workload after one warm-up step, FP64 "
                         "CPU restatement of the reference on %d threads" % (n, secs, cores)}
        # the oracle of the CPU leg has stepped the full workload from its cold start:
        # the plain FP64 library, stepped as far from the same cold start, against it
        parity = parity_vs_oracle(case, ora, ora.clock()[0])
        ora.close()

    if rank == 0:
        line = {"metric": metric, "value": value, "unit": "cell-layer updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32 fluxes, f64 state",
                "data": "synthetic", "config": cfg, "clocks": clocks, "e2e": e2e, "roofline": roof,
                "cpu_baseline": cpu, "parity": parity, "combined": combined,
                "gpu_launches": int(lib.fvg_kernels_per_step(f.h)) * args.steps}
        print(json.dumps(line), flush=True)
    f.close()
    if pg is not None:
        pg.close()


if __name__ == "__main__":
    main()
