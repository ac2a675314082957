"""The C ABI library builds for sm_100a, loads without a GPU and exports every entry
point declared in include/fvg.h (no compute call is made here)."""
import ctypes
import os
import re

from myfvcomcode_b200 import build
from myfvcomcode_b200.engine import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fvg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fvg_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.fvg_build_info.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.fvg_build_info()


def test_create_rejects_bad_arguments_without_gpu():
    lib = ctypes.CDLL(LIB_PATH)
    lib.fvg_create.restype = ctypes.c_int
    # null mesh -> FVG_ERR_ARG before any device call
    assert lib.fvg_create(None, None, None, None) == 1
