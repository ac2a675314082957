"""Generate the frozen oracle fixture of the estuary channel after 1000 external steps.

Case: the idealised estuary channel (100 x 20 structured grid split diagonally, 2,121
nodes, 4,000 cells, 10 sigma layers, M2 1.0 m, 100 m^3/s river at the head node, DTE 2 s,
ISPLIT 10).  The oracle is run from cold start for 100 internal steps (= 1000 external
steps) and the following are stored in ``channel_100x20_k10_1000ext.npz``:

* ``sha256``: digest of the float64 bytes of el, u, v, t1, s1 (ghost rows included, the
  library's Fortran-order field layout) -- pins the oracle bit for bit;
* ``el``: the full surface elevation (float64, 2,122 values);
* ``<f>_idx`` / ``<f>_val`` for u, v, t1, s1: a seeded sample of 256 interior
  (entity, layer) values each, so a device run can be compared without the oracle;
* ``<f>_layer_sum``: per-layer sums over the interior entities (numpy pairwise order).

The script is the only writer of the fixture.  Usage: ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FIXTURE = os.path.join(HERE, "channel_100x20_k10_1000ext.npz")
FIELDS = ("el", "u", "v", "t1", "s1")
SAMPLED = ("u", "v", "t1", "s1")
INTERNAL_STEPS = 100


def case():
    from myfvcomcode_b200 import cases
    return cases.estuary_channel()


def digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def summarize(engine):
    """Fixture content for the engine's current state (works for oracle and library)."""
    out = {}
    raw = {f: engine.get(f) for f in FIELDS}
    out["sha256"] = np.array(digest([raw[f] for f in FIELDS]))
    out["el"] = raw["el"]
    rng = np.random.default_rng(20240601)
    for f in SAMPLED:
        a = engine.get3(f)[1:, : engine.KB - 1]
        flat = a.reshape(-1, order="F")
        idx = np.sort(rng.choice(flat.size, size=256, replace=False))
        out[f + "_idx"] = idx.astype(np.int64)
        out[f + "_val"] = flat[idx]
        out[f + "_layer_sum"] = a.sum(axis=0)
    return out


def main():
    from oracle.oracle import Oracle
    ora = Oracle(case())
    ora.run(INTERNAL_STEPS)
    data = summarize(ora)
    np.savez_compressed(FIXTURE, **data)
    print("wrote %s sha256=%s" % (FIXTURE, str(data["sha256"])))


if __name__ == "__main__":
    main()
