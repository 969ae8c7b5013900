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
# racy-order throughput analogue (CPU baseline only): the same sources built with the sweeps over
# host threads, -O3 -march=native, on the machine that runs it
_LIB_MT = os.path.join(_HERE, "liboracle_mt.so")
_SRCS = ("oracle.cpp", "mom_ml.cpp", "mom_ke.cpp", "prep.cpp", "wind.cpp", "oracle_common.h", "oracle_ad.h", "Makefile",
         os.path.join("..", "include", "gral_prog.h"))
_lib = None
_lib_mt = None


def _make(target: str, path: str, force: bool) -> str:
    srcs = [os.path.join(_HERE, f) for f in _SRCS]
    if force or not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in srcs):
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []) + [target], check=True)
    return path


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++, no FP contraction)."""
    return _make("liboracle.so", _LIB, force)


def build_threaded(force: bool = False) -> str:
    """Compile liboracle_mt.so, the racy-order multi-threaded build (never a parity reference)."""
    return _make("liboracle_mt.so", _LIB_MT, force)


def _bind(path: str):
    h = C.CDLL(path)
    h.oracle_solve.argtypes = [C.POINTER(GralParams), C.POINTER(GralStatic),
                               C.POINTER(GralFields), C.POINTER(GralStats)]
    h.oracle_solve.restype = C.c_int
    return h


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _bind(_LIB)
    return _lib


def lib_threaded():
    global _lib_mt
    if _lib_mt is None:
        build_threaded()
        _lib_mt = _bind(_LIB_MT)
    return _lib_mt


def solve(params: dict, static: StaticArrays, fields: FieldArrays,
          trace: Optional[np.ndarray] = None, threaded: bool = False) -> dict:
    """Run the oracle in place on ``fields``; returns the stats as a dict.  ``threaded`` runs the
    racy-order multi-threaded build instead (thread count from ORACLE_THREADS, else all hardware
    threads): a throughput analogue of the reference's default mode whose results depend on thread
    timing, used only as a CPU baseline."""
    p = params_to_c(params)
    s = static.to_c()
    f = fields.to_c()
    st = GralStats()
    if trace is not None:
        st.trace_delta_umax = trace.ctypes.data_as(C.POINTER(C.c_float))
        st.trace_capacity = trace.size
    rc = (lib_threaded() if threaded else lib()).oracle_solve(C.byref(p), C.byref(s), C.byref(f), C.byref(st))
    if rc != GRAL_OK:
        raise RuntimeError(f"oracle_solve failed: {STATUS_NAMES.get(rc, rc)}")
    return stats_to_dict(st)


def threads_used() -> int:
    """Host threads the racy-order build runs its sweeps on."""
    h = lib_threaded()
    h.oracle_threads.restype = C.c_int
    return int(h.oracle_threads())


def _bind_twin(h):
    D = C.POINTER(C.c_double)
    if getattr(h, "_twin_bound", False):
        return h
    h.oracle_twin_forward.argtypes = [C.POINTER(GralParams), C.POINTER(GralStatic), C.POINTER(GralFields),
                                      D, D, D, D, C.c_int, D, D, D]
    h.oracle_twin_forward.restype = C.c_int
    h.oracle_twin_vjp.argtypes = [C.POINTER(GralParams), C.POINTER(GralStatic), C.POINTER(GralFields),
                                  D, D, D, D, C.c_int, D, D, D, D, D, D, D]
    h.oracle_twin_vjp.restype = C.c_int
    h.oracle_twin_jvp.argtypes = [C.POINTER(GralParams), C.POINTER(GralStatic), C.POINTER(GralFields),
                                  D, D, D, D, D, D, D, D, C.c_int, D, D, D]
    h.oracle_twin_jvp.restype = C.c_int
    h._twin_bound = True
    return h


def _dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def twin_forward(params: dict, static: StaticArrays, f_ref: FieldArrays, x0, veg, iterations: int):
    """FP64 twin of the model-1 path (no Frund rounding, parity width 8): `iterations` SIMPLE
    iterations from the initial fields x0 = (uk0, vk0, wk0) (float64, host layout) with vegetation
    density veg (float64, host layout, or None for the static VEG); the set-up's scalars are those
    of the reference fields f_ref.  Returns the final (uk, vk, wk) in float64."""
    p = params_to_c(params)
    s = static.to_c()
    fr = f_ref.to_c()
    uk0, vk0, wk0 = (np.ascontiguousarray(a, np.float64) for a in x0)
    vg = None if veg is None else np.ascontiguousarray(veg, np.float64)
    out = [np.zeros_like(uk0) for _ in range(3)]
    rc = _bind_twin(lib()).oracle_twin_forward(C.byref(p), C.byref(s), C.byref(fr), _dptr(uk0), _dptr(vk0),
                                               _dptr(wk0), _dptr(vg), int(iterations), *(_dptr(o) for o in out))
    if rc != GRAL_OK:
        raise RuntimeError(f"oracle_twin_forward failed: {STATUS_NAMES.get(rc, rc)}")
    return tuple(out)


def twin_vjp(params: dict, static: StaticArrays, f_ref: FieldArrays, x0, veg, iterations: int, g):
    """Reverse-mode gradient of the FP64 twin (tape differentiation of the oracle's operations):
    g = (dJ/duk, dJ/dvk, dJ/dwk) of the final fields; returns (dJ/duk0, dJ/dvk0, dJ/dwk0, dJ/dveg)."""
    p = params_to_c(params)
    s = static.to_c()
    fr = f_ref.to_c()
    uk0, vk0, wk0 = (np.ascontiguousarray(a, np.float64) for a in x0)
    vg = None if veg is None else np.ascontiguousarray(veg, np.float64)
    gu, gv, gw = (np.ascontiguousarray(a, np.float64) for a in g)
    out = [np.zeros_like(uk0) for _ in range(4)]
    rc = _bind_twin(lib()).oracle_twin_vjp(C.byref(p), C.byref(s), C.byref(fr), _dptr(uk0), _dptr(vk0), _dptr(wk0),
                                           _dptr(vg), int(iterations), _dptr(gu), _dptr(gv), _dptr(gw),
                                           *(_dptr(o) for o in out))
    if rc != GRAL_OK:
        raise RuntimeError(f"oracle_twin_vjp failed: {STATUS_NAMES.get(rc, rc)}")
    return tuple(out)


def twin_jvp(params: dict, static: StaticArrays, f_ref: FieldArrays, x0, veg, iterations: int, dx0, dveg=None):
    """Forward-mode tangent of the FP64 twin along (dx0 = (duk0, dvk0, dwk0), dveg): returns the
    derivative of the final (uk, vk, wk)."""
    p = params_to_c(params)
    s = static.to_c()
    fr = f_ref.to_c()
    a = [np.ascontiguousarray(q, np.float64) for q in x0]
    da = [np.ascontiguousarray(q, np.float64) for q in dx0]
    vg = None if veg is None else np.ascontiguousarray(veg, np.float64)
    dv = None if dveg is None else np.ascontiguousarray(dveg, np.float64)
    out = [np.zeros_like(a[0]) for _ in range(3)]
    rc = _bind_twin(lib()).oracle_twin_jvp(C.byref(p), C.byref(s), C.byref(fr), *(_dptr(q) for q in a), _dptr(vg),
                                           *(_dptr(q) for q in da), _dptr(dv), int(iterations),
                                           *(_dptr(q) for q in out))
    if rc != GRAL_OK:
        raise RuntimeError(f"oracle_twin_jvp failed: {STATUS_NAMES.get(rc, rc)}")
    return tuple(out)
