"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/fvcom_oracle.cpp).

The oracle implements the same entry-point set as the CUDA library under the ``orc_``
prefix, so tests drive both through one interface and compare fields.  Only tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from myfvcomcode_b200.engine import CEngine

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "fvcom_oracle.cpp")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_set_threads.argtypes = [C.c_int32]
        _lib.orc_set_threads.restype = C.c_int
        _lib.orc_max_threads.restype = C.c_int
        _lib.orc_set_ramp.argtypes = [C.c_void_p, C.c_double]
        _lib.orc_get_ramp.argtypes = [C.c_void_p]
        _lib.orc_get_ramp.restype = C.c_double
    return _lib


def set_threads(n):
    load().orc_set_threads(int(n))


def max_threads():
    return int(load().orc_max_threads())


class Oracle(CEngine):
    def __init__(self, case, state=None):
        super().__init__(case, load(), "orc_", state)

    def set_ramp(self, r):
        self.lib.orc_set_ramp(self.h, float(r))

    def ramp(self):
        return self.lib.orc_get_ramp(self.h)
