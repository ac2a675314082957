"""Error of the precision form against the plain FP64 path after a simulated period.

Both forms start from the same cold start of the same case and run the same number of
internal steps on the device.  Reported per output (zeta, u, v, T, S): the maximum and
RMS absolute difference over the interior entities and layers, and for each form the
drift of the volume, heat and salt budgets (``fvg_budget``) over the run.  The controls
"fp64_twin" and "fp64_twin2" are FP64 again from initial temperatures perturbed by 1e-6 C
(two seeds): their differences from FP64 are what perturbations of the size of FP32
rounding grow to by themselves in this flow.

    python -m myfvcomcode_b200.precision_report [--npts 200000] [--hours 24] [--md FILE] [--json FILE]

The form with the learned closure ("fp32flux_learned") is run beside the precision form
alone, with the network the library ships (trained on the 50k-node coastal mesh).
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import json
import math
import os
import subprocess
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def sources_stamp():
    """sha256 over everything the report's numbers depend on: the CUDA sources, the C-ABI
    header, and the host code that builds the case and its mesh metrics."""
    files = sorted(glob.glob(os.path.join(_HERE, "csrc", "*.cu")) + glob.glob(os.path.join(_HERE, "csrc", "*.h")))
    files += [os.path.join(_HERE, "..", "include", "fvg.h")]
    files += [os.path.join(_HERE, n) for n in ("cases.py", "grid.py", "startup.py", "abi.py", "build.py")]
    h = hashlib.sha256()
    for fn in files:
        h.update(os.path.basename(fn).encode())
        with open(fn, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _commit():
    try:
        return subprocess.run(["git", "-C", _HERE, "rev-parse", "--short=12", "HEAD"], capture_output=True,
                              text=True, timeout=10).stdout.strip() or None
    except Exception:
        return None


def _interior(engine, name):
    if name == "el":
        return engine.get("el")[1:]
    return engine.get3(name)[1:, : engine.KB - 1]


def compare(ref, other):
    out = {}
    for name, label in (("el", "zeta_m"), ("u", "u_m_s"), ("v", "v_m_s"), ("t1", "T_C"), ("s1", "S_psu")):
        a, b = _interior(ref, name), _interior(other, name)
        d = np.abs(a - b)
        out[label] = {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d)))}
    return out


def twin_case(case, amplitude=1e-6, seed=17):
    """``case`` with the initial temperature perturbed by N(0, amplitude) per node: the
    control that measures how far FP64 runs drift apart from differences of the size of
    FP32 rounding alone."""
    c = dict(case)
    c["init"] = dict(case["init"])
    rng = np.random.default_rng(seed)
    off = rng.normal(0.0, amplitude, case["grid"]["M"] + 1)
    off[0] = 0.0
    c["init"]["t_offset"] = off
    return c


TWIN_SEEDS = {"fp64_twin": 17, "fp64_twin2": 29}
# the learned closure of the chosen form: the network trained on the 50k-node coastal mesh
LEARNED = os.path.join(_HERE, "data", "closure_coastal50k_8seeds.npz")


def run(case, steps, modes=("fp64", "fp32flux", "fp32flux_learned", "fp64_twin", "fp64_twin2"), chunk=200):
    """Every mode from the same cold start for ``steps`` internal steps: "fp32flux" the
    precision form, "fp32flux_learned" the precision form with the learned closure (MY2.5
    as its per-column fallback); the twins are FP64 from initial temperatures perturbed by
    1e-6 C with different seeds (their spread shows how far this flow's own sensitivity
    alone moves the fields)."""
    from . import closure
    from .engine import Fvcom
    engines = {}
    budgets = {}
    times = {}
    for m in modes:
        twin = m in TWIN_SEEDS
        f = Fvcom(twin_case(case, seed=TWIN_SEEDS[m]) if twin else case)
        f.set_precision("fp64" if twin else ("fp32flux" if m == "fp32flux_learned" else m))
        if m == "fp32flux_learned":
            closure.attach(f, closure.load(LEARNED))
        b0 = f.budget()
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            f.run(n)
            done += n
            if f.shutdown_check() != 0:
                raise RuntimeError("%s: non-finite state after %d steps" % (m, done))
        f.sync()
        times[m] = time.perf_counter() - t0
        b1 = f.budget()
        budgets[m] = {k: (b1[i] - b0[i]) / b0[i] if b0[i] != 0 else math.nan
                      for i, k in enumerate(("volume", "heat", "salt"))}
        engines[m] = f
    ref = engines[modes[0]]
    report = {"case": case["name"], "internal_steps": steps, "sources_sha256": sources_stamp(),
              "commit": _commit(),
              "simulated_hours": steps * case["params"]["DTE"] * case["params"]["ISPLIT"] / 3600.0,
              "budget_drift": budgets, "wall_s": times, "errors_vs_" + modes[0]: {}}
    for m in modes[1:]:
        report["errors_vs_" + modes[0]][m] = compare(ref, engines[m])
    for f in engines.values():
        f.close()
    return report


def markdown(rep):
    lines = ["| output (form) | max abs difference from FP64 | RMS difference |", "|---|---|---|"]
    for m, errs in rep["errors_vs_fp64"].items():
        for k, v in errs.items():
            lines.append("| %s (%s) | %.3e | %.3e |" % (k, m, v["max"], v["rms"]))
    lines.append("")
    lines.append("| form | volume drift | heat drift | salt drift |")
    lines.append("|---|---|---|---|")
    for m, b in rep["budget_drift"].items():
        lines.append("| %s | %.3e | %.3e | %.3e |" % (m, b["volume"], b["heat"], b["salt"]))
    return "\n".join(lines) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--npts", type=int, default=200000)
    ap.add_argument("--hours", type=float, default=24.0)
    ap.add_argument("--md", default=None)
    ap.add_argument("--json", default=None, help="also write the report to this file")
    args = ap.parse_args()
    from . import cases
    case = cases.coastal_mesh(npts=args.npts)
    dti = case["params"]["DTE"] * case["params"]["ISPLIT"]
    steps = int(round(args.hours * 3600.0 / dti))
    rep = run(case, steps)
    print(json.dumps(rep))
    if args.json:
        with open(args.json, "w") as fh:
            json.dump(rep, fh)
    if args.md:
        with open(args.md, "w") as fh:
            fh.write(markdown(rep))


if __name__ == "__main__":
    main()
