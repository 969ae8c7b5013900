"""TEST INFRASTRUCTURE ONLY: Python entry to the oracle's restatement of the flow-field set-up
(``prep.cpp`` in ``liboracle.so``): prognostic sub-domains, flat-terrain initial field with its
near-wall damping, vegetation rasterisation.  Used by the tests and the CPU legs of bench.py as
the checker of ``gral_prog_subdomains``, ``gral_prog_flat_init`` and ``gral_prog_vegetation``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gral_b200.abi import (PARTICLE_DTYPE, FieldArrays, GralFields, GralFlatGrid, GralMet, GralVegPoint,
                           GralWindGrid, MetProfile, veg_points_to_c)

from . import oracle as _o

_ready = False


def _lib():
    global _ready
    L = _o.lib()
    if not _ready:
        vp = C.c_void_p
        L.oracle_subdomains.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, vp, vp]
        L.oracle_subdomains.restype = None
        L.oracle_flat_init.argtypes = [C.POINTER(GralFlatGrid), vp, vp, vp, vp, C.POINTER(GralMet), vp, vp,
                                       C.POINTER(C.c_int32), C.POINTER(GralFields)]
        L.oracle_flat_init.restype = C.c_int
        L.oracle_vegetation.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, C.POINTER(GralVegPoint),
                                        vp, vp, vp]
        L.oracle_vegetation.restype = None
        L.oracle_wind_at.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(GralWindGrid), vp, vp, vp, vp, vp,
                                     C.c_int, vp, vp, vp, vp, vp]
        L.oracle_wind_at.restype = None
        _ready = True
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def subdomains(cutk, nii, njj, dxk, dyk, factor=15):
    """ADVDOM of ReadGeometryAndDomains.cs:321-347."""
    cutk = _f32(cutk)
    adv = np.zeros((nii + 2, njj + 2), np.uint8)
    _lib().oracle_subdomains(nii, njj, dxk, dyk, factor, cutk.ctypes.data, adv.ctypes.data)
    return adv


def flat_init(grid: dict, cutk, dzk, hokart, met: MetProfile, advdom=None):
    """MicroscaleFlat.cs:29-357 in its sequential order; returns (kkart, ahk, kadvmax, fields)."""
    nii, njj, nkk = grid["nii"], grid["njj"], grid["nkk"]
    g = GralFlatGrid(**grid)
    cutk, dzk, hokart = _f32(cutk), _f32(dzk), _f32(hokart)
    adv = None if advdom is None else np.ascontiguousarray(advdom, np.uint8)
    shape = (nii + 2, njj + 2, nkk + 2)
    f = FieldArrays(*(np.zeros(shape, np.float32) for _ in range(3)))
    kk = np.zeros((nii + 2, njj + 2), np.int16)
    ahk = np.zeros((nii + 2, njj + 2), np.float32)
    kadv = C.c_int32()
    m = met.to_c()
    fc = f.to_c()
    rc = _lib().oracle_flat_init(C.byref(g), cutk.ctypes.data, dzk.ctypes.data, hokart.ctypes.data,
                                 None if adv is None else adv.ctypes.data, C.byref(m), kk.ctypes.data,
                                 ahk.ctypes.data, C.byref(kadv), C.byref(fc))
    if rc != 0:
        raise RuntimeError(f"oracle_flat_init failed: {rc}")
    return kk, ahk, kadv.value, f


def vegetation(nii, njj, nkk, kkart, dzk, hokart, points, cov):
    """VEG, the allocation mask and COV after ReadVegetation.cs:83-118 (cov: values before)."""
    veg = np.zeros((nii + 2, njj + 2, nkk + 2), np.float32)
    mask = np.zeros((nii + 2, njj + 2), np.uint8)
    cov = _f32(cov).copy()
    kk = np.ascontiguousarray(kkart, np.int16)
    dz, ho = _f32(dzk), _f32(hokart)
    pts = veg_points_to_c(points)
    _lib().oracle_vegetation(nii, njj, nkk, kk.ctypes.data, dz.ctypes.data, ho.ctypes.data,
                             len(points), pts, veg.ctypes.data, mask.ctypes.data, cov.ctypes.data)
    return veg, mask, cov


def wind_at(grid: dict, nii, njj, nkk, dzk, hokart, fields, particles, met: MetProfile = None):
    """IntWindCalculate (Intwind.cs:31-197) per particle; returns (ux, uy, uz, index_k)."""
    p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
    n = p.size
    ux, uy, uz = (np.zeros(n, np.float32) for _ in range(3))
    kk = np.zeros(n, np.int32)
    m = None if met is None else met.to_c()
    g = GralWindGrid(grid.get("terrain", 0), grid.get("buildings", 1), grid.get("ikooa", 0), grid.get("jkooa", 0),
                     grid["dxk"], grid["dyk"], grid.get("ahmin", 0.0),
                     C.pointer(m) if m is not None else C.POINTER(GralMet)())
    dz = _f32(dzk) if dzk is not None else np.zeros(nkk + 2, np.float32)
    ho = _f32(hokart) if hokart is not None else np.zeros(nkk + 2, np.float32)
    u, v, w = (_f32(a) for a in (fields.uk, fields.vk, fields.wk)) if fields is not None else \
        (np.zeros(1, np.float32),) * 3
    _lib().oracle_wind_at(nii, njj, nkk, C.byref(g), dz.ctypes.data, ho.ctypes.data, u.ctypes.data, v.ctypes.data,
                          w.ctypes.data, n, p.ctypes.data, ux.ctypes.data, uy.ctypes.data, uz.ctypes.data,
                          kk.ctypes.data)
    return ux, uy, uz, kk

