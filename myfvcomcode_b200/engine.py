"""Host-side mirror of FVCOM's time-step interface over the C ABI (include/fvg.h).

``Fvcom(case)`` owns one library handle: the mesh goes to the device once, the
cold-start state is copied in, and ``internal_step()`` / ``run(n)`` advance the model
exactly as fvcom.F:848-852 calls INTERNAL_STEP.  ``routine(r, arg)`` runs one reference
subroutine (enum fvg_routine) for per-routine parity checks; ``get``/``set`` move any
FVCOM variable by its (lower-case) name.

The CUDA library is required: if libfvg.so is missing or fails to load, construction
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .startup import coldstart

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfvg.so")

ROUTINES = dict(
    EXTEL_EDGE=1, BCOND_ELF=2, N2E2D_ELF=3, WET_JUDGE=4, FLUX_OBN=5, ADVAVE=6, EXTUV_EDGE=7,
    BCOND_UV2D=8, EXT_UPDATE=9, EXTERNAL_STEP=10, ADJUST2D3D=11, BCOND_UV3D_SOLID=12,
    BROUGH=13, ADVECTION3D=14, BAROPG=15, INT_PRE_EXT=16, VERTVL=17, VISCOFH=18, ADV_UV=19,
    VDIF_UV=20, BCOND_UV3D=21, WREAL=22, ADV_Q=23, FCT_Q=24, VDIF_Q=25, TURB_UPDATE=26,
    ADV_TS=27, FCT_TS=28, VDIF_TS=29, BCOND_TS=30, TS_UPDATE=31, DENS2=32, INT_FINAL=33,
    INTERNAL_STEP=34, INT_FORCING=35,
)

INT_FIELDS = ("iswetn", "iswetnt", "iswetc", "iswetct", "iswetce")


class FvgError(RuntimeError):
    pass


def _declare(lib, prefix):
    P = C.POINTER
    vp = C.c_void_p
    fn = lambda n: getattr(lib, prefix + n)
    fn("create").argtypes = [P(abi.FvgMesh), P(abi.FvgParams), P(abi.FvgForcing), P(vp)]
    fn("create").restype = C.c_int
    fn("destroy").argtypes = [vp]
    fn("destroy").restype = None
    for n, t in (("set_field", P(C.c_double)), ("get_field", P(C.c_double)),
                 ("set_ifield", P(C.c_int32)), ("get_ifield", P(C.c_int32))):
        fn(n).argtypes = [vp, C.c_char_p, t, C.c_int64]
        fn(n).restype = C.c_int
    fn("field_size").argtypes = [vp, C.c_char_p]
    fn("field_size").restype = C.c_int64
    fn("set_clock").argtypes = [vp, C.c_int32, C.c_double]
    fn("set_clock").restype = C.c_int
    fn("get_clock").argtypes = [vp, P(C.c_int32), P(C.c_double)]
    fn("get_clock").restype = C.c_int
    fn("internal_step").argtypes = [vp]
    fn("internal_step").restype = C.c_int
    fn("run").argtypes = [vp, C.c_int32]
    fn("run").restype = C.c_int
    fn("run_routine").argtypes = [vp, C.c_int32, C.c_int32]
    fn("run_routine").restype = C.c_int


class CEngine:
    """Generic driver of a C library that implements the fvg_* entry-point set."""

    prefix = "fvg_"

    def __init__(self, case, lib, prefix=None, state=None):
        self.prefix = prefix or self.prefix
        self.lib = lib
        _declare(lib, self.prefix)
        self.case = case
        g = case["grid"]
        self.M, self.N, self.KB = g["M"], g["N"], g["KB"]
        self._ms, self._ps, self._fs, self._bundle = abi.make_structs(case)
        h = C.c_void_p()
        rc = self._f("create")(C.byref(self._ms), C.byref(self._ps), C.byref(self._fs), C.byref(h))
        self._check(rc, "create", handle=False)
        self.h = h
        self.set_state(coldstart(case) if state is None else state)

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, rc, what, handle=True):
        if rc != 0:
            msg = ""
            if handle and hasattr(self.lib, self.prefix + "last_error"):
                f = self._f("last_error")
                f.restype = C.c_char_p
                f.argtypes = [C.c_void_p]
                m = f(self.h)
                msg = m.decode() if m else ""
            raise FvgError("%s%s failed with status %d %s" % (self.prefix, what, rc, msg))

    def size(self, name):
        return int(self._f("field_size")(self.h, name.encode()))

    def get(self, name):
        n = self.size(name)
        if n < 0:
            raise KeyError(name)
        if name in INT_FIELDS:
            out = np.zeros(n, dtype=np.int32)
            rc = self._f("get_ifield")(self.h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_int32)), n)
        else:
            out = np.zeros(n, dtype=np.float64)
            rc = self._f("get_field")(self.h, name.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), n)
        self._check(rc, "get_field(%s)" % name)
        return out

    def get3(self, name):
        a = self.get(name)
        rows = a.size // self.KB
        return a.reshape((rows, self.KB), order="F")

    def set(self, name, arr):
        if name in INT_FIELDS:
            a = np.ascontiguousarray(np.asarray(arr, dtype=np.int32).reshape(-1, order="F"))
            rc = self._f("set_ifield")(self.h, name.encode(), a.ctypes.data_as(C.POINTER(C.c_int32)), a.size)
        else:
            a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64).reshape(-1, order="F"))
            rc = self._f("set_field")(self.h, name.encode(), a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        self._check(rc, "set_field(%s)" % name)

    def set_state(self, st):
        for k, v in st.items():
            self.set(k, v)

    def clock(self):
        i = C.c_int32()
        t = C.c_double()
        self._check(self._f("get_clock")(self.h, C.byref(i), C.byref(t)), "get_clock")
        return i.value, t.value

    def set_clock(self, iint, ext_time):
        self._check(self._f("set_clock")(self.h, int(iint), float(ext_time)), "set_clock")

    def internal_step(self):
        self._check(self._f("internal_step")(self.h), "internal_step")

    def set_forcing(self, forcing):
        """Replace the boundary forcing between internal steps (fvg_set_forcing):
        ``forcing`` has the keys of ``case["forcing"]`` (tide, qdis, tdis, sdis, wind);
        the tide must keep its number of constituents, and wind needs a model created
        with wind."""
        fs = abi.forcing_struct(dict(self.case, forcing=forcing))
        f = self._f("set_forcing")
        f.argtypes = [C.c_void_p, C.c_void_p]
        f.restype = C.c_int
        self._check(f(self.h, C.byref(fs)), "set_forcing")

    def run(self, n):
        self._check(self._f("run")(self.h, int(n)), "run")

    def routine(self, name, arg=0):
        r = ROUTINES[name] if isinstance(name, str) else int(name)
        self._check(self._f("run_routine")(self.h, r, int(arg)), "run_routine(%s)" % name)

    def close(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_LIB = None


def load_library(path=None):
    """Load the in-tree CUDA library; raise if it is absent (no fallback exists)."""
    global _LIB
    if _LIB is None:
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise FvgError("libfvg.so not built at %s (run __graft_entry__.build())" % p)
        _LIB = C.CDLL(p)
    return _LIB


class Fvcom(CEngine):
    """The B200 mode-split step for one model (mesh + parameters + forcing)."""

    def __init__(self, case, state=None, lib_path=None):
        lib = load_library(lib_path)
        super().__init__(case, lib, "fvg_", state)

    def sync(self):
        self._check(self.lib.fvg_sync(self.h), "sync")

    def set_ramp(self, r):
        self.lib.fvg_set_ramp.argtypes = [C.c_void_p, C.c_double]
        self._check(self.lib.fvg_set_ramp(self.h, float(r)), "set_ramp")

    def use_graph(self, on):
        self.lib.fvg_use_graph.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.fvg_use_graph(self.h, int(bool(on))), "use_graph")

    def budget(self):
        out = (C.c_double * 3)()
        self.lib.fvg_budget.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        self._check(self.lib.fvg_budget(self.h, out), "budget")
        return tuple(out)

    def shutdown_check(self):
        return int(self.lib.fvg_shutdown_check(self.h))

    PRECISION = {"fp64": 0, "fp32flux": 1}

    def set_precision(self, mode):
        """'fp64' (plain, bitwise equal to the oracle) or 'fp32flux' (FP32 edge fluxes and
        advection, FP64 elevation update, column solves, state and budgets)."""
        m = self.PRECISION[mode] if isinstance(mode, str) else int(mode)
        self.lib.fvg_set_precision.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.fvg_set_precision(self.h, m), "set_precision")

    def get_precision(self):
        self.lib.fvg_get_precision.argtypes = [C.c_void_p]
        self.lib.fvg_get_precision.restype = C.c_int32
        return {v: k for k, v in self.PRECISION.items()}[self.lib.fvg_get_precision(self.h)]

    def set_tuning(self, key, value):
        self.lib.fvg_set_tuning.argtypes = [C.c_void_p, C.c_char_p, C.c_int32]
        self._check(self.lib.fvg_set_tuning(self.h, key.encode(), int(value)), "set_tuning(%s)" % key)

    def get_tuning(self, key):
        v = C.c_int32()
        self.lib.fvg_get_tuning.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]
        self._check(self.lib.fvg_get_tuning(self.h, key.encode(), C.byref(v)), "get_tuning(%s)" % key)
        return v.value

    def time_steps(self, n):
        """Run n internal steps; device milliseconds (CUDA events on the handle's stream)."""
        ms = C.c_double()
        self.lib.fvg_time_steps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        self._check(self.lib.fvg_time_steps(self.h, int(n), C.byref(ms)), "time_steps")
        return ms.value


class Group:
    """Several Fvcom models stepped together by one CUDA graph per internal step."""

    def __init__(self, models):
        self.models = list(models)
        self.lib = self.models[0].lib
        arr = (C.c_void_p * len(self.models))(*[m.h for m in self.models])
        g = C.c_void_p()
        self.lib.fvg_group_create.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]
        rc = self.lib.fvg_group_create(arr, len(self.models), C.byref(g))
        if rc != 0:
            raise FvgError("fvg_group_create failed with status %d" % rc)
        self.g = g

    def _check(self, rc, what):
        if rc != 0:
            self.lib.fvg_group_last_error.argtypes = [C.c_void_p]
            self.lib.fvg_group_last_error.restype = C.c_char_p
            raise FvgError("%s failed with status %d %s" % (what, rc, self.lib.fvg_group_last_error(self.g).decode()))

    def run(self, n):
        self.lib.fvg_group_run.argtypes = [C.c_void_p, C.c_int32]
        self._check(self.lib.fvg_group_run(self.g, int(n)), "fvg_group_run")

    def time_steps(self, n):
        ms = C.c_double()
        self.lib.fvg_group_time_steps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
        self._check(self.lib.fvg_group_time_steps(self.g, int(n), C.byref(ms)), "fvg_group_time_steps")
        return ms.value

    def close(self):
        if getattr(self, "g", None):
            self.lib.fvg_group_destroy.argtypes = [C.c_void_p]
            self.lib.fvg_group_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """The learned closure's network (fvg_mlp_*): parameters on the device, trained by the
    library's CUDA kernels.  Data arguments are device pointers (ints) to float32 arrays."""

    def __init__(self, seed=0, lib_path=None):
        self.lib = load_library(lib_path)
        L = self.lib
        L.fvg_mlp_create.argtypes = [C.c_uint64, C.POINTER(C.c_void_p)]
        L.fvg_mlp_destroy.argtypes = [C.c_void_p]
        L.fvg_mlp_last_error.argtypes = [C.c_void_p]
        L.fvg_mlp_last_error.restype = C.c_char_p
        L.fvg_mlp_num_params.restype = C.c_int32
        fp = C.POINTER(C.c_float)
        L.fvg_mlp_get_params.argtypes = [C.c_void_p, fp, C.c_int32]
        L.fvg_mlp_set_params.argtypes = [C.c_void_p, fp, C.c_int32]
        L.fvg_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, fp, fp]
        L.fvg_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_float, C.c_uint64, fp]
        L.fvg_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        L.fvg_mlp_device_params.argtypes = [C.c_void_p]
        L.fvg_mlp_device_params.restype = C.c_void_p
        h = C.c_void_p()
        rc = L.fvg_mlp_create(int(seed), C.byref(h))
        if rc != 0:
            raise FvgError("fvg_mlp_create failed with status %d" % rc)
        self.h = h
        self.npar = int(L.fvg_mlp_num_params())

    def _check(self, rc, what):
        if rc != 0:
            raise FvgError("%s failed with status %d %s" % (what, rc, self.lib.fvg_mlp_last_error(self.h).decode()))

    def params(self):
        out = np.zeros(self.npar, dtype=np.float32)
        self._check(self.lib.fvg_mlp_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), self.npar),
                    "fvg_mlp_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.lib.fvg_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), self.npar),
                    "fvg_mlp_set_params")

    def loss_grad(self, x_ptr, y_ptr, n):
        loss = C.c_float()
        g = np.zeros(self.npar, dtype=np.float32)
        self._check(self.lib.fvg_mlp_loss_grad(self.h, x_ptr, y_ptr, int(n), C.byref(loss),
                                               g.ctypes.data_as(C.POINTER(C.c_float))), "fvg_mlp_loss_grad")
        return loss.value, g

    def train(self, x_ptr, y_ptr, n, epochs, batch, lr, seed=0):
        hist = np.zeros(epochs, dtype=np.float32)
        self._check(self.lib.fvg_mlp_train(self.h, x_ptr, y_ptr, int(n), int(epochs), int(batch), float(lr),
                                           int(seed), hist.ctypes.data_as(C.POINTER(C.c_float))), "fvg_mlp_train")
        return hist

    def forward(self, x_ptr, n, out_ptr):
        self._check(self.lib.fvg_mlp_forward(self.h, x_ptr, int(n), out_ptr), "fvg_mlp_forward")

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
