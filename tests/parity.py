"""Helpers shared by the parity tests: field lists, state transfer and comparison.

Two measures of a difference between the library's field ``a`` and the oracle's ``b``:

* max-normalised: max|a - b| / max|b| over the field (``compare``'s ``rtol``), a norm
  that grants every element the field's largest magnitude;
* per element: max over elements of |a_i - b_i| / max(|b_i|, 1e-6 max|b|), i.e. each
  element's own relative error, with elements below a millionth of the field's scale
  held to that floor instead of their own (near-zero) size (``errors``).
"""
from __future__ import annotations

import numpy as np

NODE2 = ["el", "elf", "elrk", "et", "d", "dt", "dtfa", "egf", "wubot_n", "wvbot_n", "taubm_n"]
NODE3 = ["t1", "s1", "tf1", "sf1", "rho1", "tmean1", "smean1", "rmean1", "q2", "q2l", "q2f",
         "q2lf", "l", "km", "kh", "kq", "wts", "viscofh"]
CELL2 = ["el1", "elf1", "elrk1", "et1", "d1", "dt1", "ua", "va", "uaf", "vaf", "uark", "vark",
         "uard", "vard", "adx2d", "ady2d", "drx2d", "dry2d", "advua", "advva", "pstx", "psty",
         "wubot", "wvbot", "cbc", "tps", "fluxobn", "taubm", "wusurf", "wvsurf"]
CELL3 = ["u", "v", "uf", "vf", "w", "ww", "advx", "advy", "drhox", "drhoy", "rho", "t", "s",
         "rmean", "km1", "viscofm"]
INTS = ["iswetn", "iswetnt", "iswetc", "iswetct", "iswetce"]
OTHER = ["xflux_obcn", "uard_obcn", "qdis"]
# oracle name -> names of the CUDA library's per-tracer copies
MAPPED = {"pfpxb": ("pfpxb_t", "pfpxb_s"), "pfpyb": ("pfpyb_t", "pfpyb_s"),
          "ah_bottom": ("ah_bottom_t", "ah_bottom_s"), "xflux_obc": ("xflux_obc_t", "xflux_obc_s")}
ALL = NODE2 + NODE3 + CELL2 + CELL3 + INTS + OTHER


def copy_state(src, dst):
    """Copy every state field from the oracle ``src`` to the library ``dst``."""
    for n in ALL:
        dst.set(n, src.get(n))
    for o, (a, b) in MAPPED.items():
        v = src.get(o)
        dst.set(a, v)
        dst.set(b, v)
    i, t = src.clock()
    dst.set_clock(i, t)
    dst.set_ramp(src.ramp())


def copy_oracle_state(src, dst):
    """Copy every state field between two oracles (their own field names)."""
    for n in ALL + list(MAPPED):
        dst.set(n, src.get(n))
    i, t = src.clock()
    dst.set_clock(i, t)
    dst.set_ramp(src.ramp())


def gpu_name(name, tracer=1):
    if name in MAPPED:
        return MAPPED[name][tracer - 1]
    return name


def interior(engine, name, arr):
    """Drop the ghost row 0 of every layer."""
    KB = engine.KB
    n = arr.size
    rows = n
    for lay in (KB, KB - 1):
        for L in (engine.M + 1, engine.N + 1):
            if n == L * lay and lay > 1:
                return arr.reshape((L, lay), order="F")[1:]
    return arr[1:]


def compare(gpu, ora, names, rtol=0.0, tracer=1):
    """Return {name: max relative difference}; rtol == 0 demands bitwise equality."""
    bad = {}
    for n in names:
        a = interior(gpu, n, gpu.get(gpu_name(n, tracer)))
        b = interior(ora, n, ora.get(n))
        if rtol == 0.0:
            if not np.array_equal(a, b, equal_nan=True):
                diff = np.abs(a.astype(np.float64) - b.astype(np.float64))
                bad[n] = float(np.nanmax(diff)) if diff.size else 0.0
        else:
            scale = max(float(np.abs(b).max()) if b.size else 0.0, 1e-30)
            d = float(np.abs(a - b).max()) / scale if b.size else 0.0
            if not d <= rtol:
                bad[n] = d
    return bad


def errors(gpu, ora, names, tracer=1):
    """{name: {"max_norm": ..., "per_element": ..., "bitwise": bool}} for ``names``."""
    out = {}
    for n in names:
        a = interior(gpu, n, gpu.get(gpu_name(n, tracer))).astype(np.float64)
        b = interior(ora, n, ora.get(n)).astype(np.float64)
        d = np.abs(a - b)
        scale = float(np.abs(b).max()) if b.size else 0.0
        floor = max(1e-6 * scale, 1e-300)
        out[n] = {"max_norm": float(d.max()) / max(scale, 1e-300) if b.size else 0.0,
                  "per_element": float((d / np.maximum(np.abs(b), floor)).max()) if b.size else 0.0,
                  "bitwise": bool(np.array_equal(a, b, equal_nan=True))}
    return out
