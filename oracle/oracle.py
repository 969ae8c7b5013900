"""TEST INFRASTRUCTURE ONLY: ctypes loader of the CPU oracle (``liboracle.so``).

The oracle restates GRAL's deterministic prognostic solve (see oracle_common.h); only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it, as the checker.
Parity unpinned: the C# reference cannot run here and ships no golden vectors for this path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from gral_b200.abi import (GralFields, GralParams, GralStatic, GralStats, FieldArrays,
                           StaticArrays, params_to_c, stats_to_dict, GRAL_OK, STATUS_NAMES)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++, no FP contraction)."""
    srcs = [os.path.join(_HERE, f) for f in ("oracle.cpp", "mom_ml.cpp", "mom_ke.cpp", "prep.cpp", "wind.cpp", "oracle_common.h",
                                              os.path.join("..", "include", "gral_prog.h"))]
    if force or not os.path.exists(_LIB) or any(os.path.getmtime(s) > os.path.getmtime(_LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
        _lib.oracle_solve.argtypes = [C.POINTER(GralParams), C.POINTER(GralStatic),
                                      C.POINTER(GralFields), C.POINTER(GralStats)]
        _lib.oracle_solve.restype = C.c_int
    return _lib


def solve(params: dict, static: StaticArrays, fields: FieldArrays,
          trace: Optional[np.ndarray] = None) -> dict:
    """Run the oracle in place on ``fields``; returns the stats as a dict."""
    p = params_to_c(params)
    s = static.to_c()
    f = fields.to_c()
    st = GralStats()
    if trace is not None:
        st.trace_delta_umax = trace.ctypes.data_as(C.POINTER(C.c_float))
        st.trace_capacity = trace.size
    rc = lib().oracle_solve(C.byref(p), C.byref(s), C.byref(f), C.byref(st))
    if rc != GRAL_OK:
        raise RuntimeError(f"oracle_solve failed: {STATUS_NAMES.get(rc, rc)}")
    return stats_to_dict(st)
