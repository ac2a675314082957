"""Launch-shape autotuner of the column-tiled 3-D kernels.

The 3-D gather kernels run one thread per cell or node walking ``col_layers`` consecutive
layers, ``col_threads`` threads per block (``fvg_set_tuning``).  Their results do not
depend on the shape, so the tuner times candidate shapes and returns the fastest.

Without ``engine`` the candidates run on a throw-away handle of the same case, and no
model of the caller's is advanced.  With ``engine=f`` they run on ``f`` itself, which is
advanced by (warmup + steps) internal steps per candidate; callers that compare forms
(``bench.py``) tune every handle the same way so that they stay step for step alike.
"""
from __future__ import annotations

import itertools

DEFAULT_THREADS = (64, 128, 256)
DEFAULT_LAYERS = (1, 2, 4, 8, 20, 40)


def candidates(kb, threads=DEFAULT_THREADS, layers=DEFAULT_LAYERS):
    ls = sorted({min(l, kb) for l in layers})
    return list(itertools.product(threads, ls))


def autotune(case, cands=None, steps=3, warmup=1, engine=None):
    """Time each (col_threads, col_layers) over ``steps`` internal steps after ``warmup``.

    Returns {"col_threads", "col_layers", "ms_per_step", "table": [(ms, threads, layers)]}.
    """
    from .engine import Fvcom
    fv = engine if engine is not None else Fvcom(case)
    try:
        table = []
        for bc, lc in (cands or candidates(fv.KB)):
            fv.set_tuning("col_threads", bc)
            fv.set_tuning("col_layers", lc)
            fv.time_steps(warmup)
            table.append((fv.time_steps(steps) / steps, bc, lc))
        ms, bc, lc = min(table)
        return {"col_threads": bc, "col_layers": lc, "ms_per_step": ms, "table": table}
    finally:
        if engine is None:
            fv.close()


def apply(fv, tuned):
    fv.set_tuning("col_threads", tuned["col_threads"])
    fv.set_tuning("col_layers", tuned["col_layers"])
