"""ctypes mirror of ``include/gral_prog.h``.

The structs below follow the C header field by field; ``tests/test_abi.py`` checks their sizes
against the compiled library.  Helpers turn numpy arrays into the pointer structs without
copying (the caller keeps the arrays alive for the duration of a call).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

ABI_VERSION = 1

GRAL_OK = 0
GRAL_EINVAL = -1
GRAL_ENOMEM = -2
GRAL_ECUDA = -3
GRAL_ETIMEDOUT = -4
GRAL_ENONFINITE = -5
GRAL_ENODEV = -6
GRAL_ESTATE = -7
GRAL_ETOOLARGE = -8
GRAL_NOALLOC_MAX_ROWS = 4096

STATUS_NAMES = {
    GRAL_OK: "GRAL_OK", GRAL_EINVAL: "GRAL_EINVAL", GRAL_ENOMEM: "GRAL_ENOMEM",
    GRAL_ECUDA: "GRAL_ECUDA", GRAL_ETIMEDOUT: "GRAL_ETIMEDOUT",
    GRAL_ENONFINITE: "GRAL_ENONFINITE", GRAL_ENODEV: "GRAL_ENODEV", GRAL_ESTATE: "GRAL_ESTATE",
    GRAL_ETOOLARGE: "GRAL_ETOOLARGE",
}

MAX_HISTORY = 64

_fp = C.POINTER(C.c_float)
_i16p = C.POINTER(C.c_int16)
_u8p = C.POINTER(C.c_uint8)


class GralParams(C.Structure):
    _fields_ = [
        ("nii", C.c_int32), ("njj", C.c_int32), ("nkk", C.c_int32),
        ("kadvmax", C.c_int32), ("vert_cells_ff", C.c_int32),
        ("dxk", C.c_float), ("dyk", C.c_float),
        ("turbulence_model", C.c_int32), ("simd_width", C.c_int32),
        ("iteration_steps_min", C.c_int32), ("iteration_steps_max", C.c_int32),
        ("conv_cadence", C.c_int32), ("conv_threshold", C.c_double),
        ("relax", C.c_float), ("relaxp", C.c_float),
        ("building_z0", C.c_float), ("coriolis", C.c_float), ("potdtdz", C.c_float),
        ("ref_i", C.c_int32), ("ref_j", C.c_int32),
        ("quantise", C.c_int32), ("turb_init", C.c_int32),
        ("std_dev_v", C.c_float), ("std_dev_w", C.c_float),
        ("bd_lay_height", C.c_float), ("v0_1", C.c_float),
        ("post_diagnostic", C.c_int32),
    ]


class GralStatic(C.Structure):
    _fields_ = [
        ("kkart", _i16p), ("advdom", _u8p), ("cutk", _fp), ("cov", _fp), ("z0", _fp),
        ("z0_init", _fp), ("ob_init", _fp), ("ust_init", _fp),
        ("veg", _fp), ("veg_mask", _u8p), ("dzk", _fp), ("hokart", _fp),
    ]


class GralFields(C.Structure):
    _fields_ = [("uk", _fp), ("vk", _fp), ("wk", _fp), ("turb", _fp), ("tdiss", _fp)]


class GralMet(C.Structure):
    _fields_ = [("n_heights", C.c_int32), ("measurement_height", _fp), ("obs_u", _fp), ("obs_v", _fp),
                ("ob_length", C.c_float), ("ol_column", _fp)]


class GralFlatGrid(C.Structure):
    _fields_ = [("nii", C.c_int32), ("njj", C.c_int32), ("nkk", C.c_int32), ("vert_cells_ff", C.c_int32),
                ("dxk", C.c_float), ("dyk", C.c_float), ("near_wall", C.c_int32), ("igeb", C.c_int32)]


class GralVegPoint(C.Structure):
    _fields_ = [("crown_height", C.c_double), ("trunk_height", C.c_double), ("trunk_lad", C.c_double),
                ("crown_lad", C.c_double), ("cov", C.c_double), ("i", C.c_int32), ("j", C.c_int32),
                ("drag", C.c_int32), ("reserved", C.c_int32)]


class GralWindGrid(C.Structure):
    _fields_ = [("terrain", C.c_int32), ("buildings", C.c_int32), ("ikooa", C.c_int32), ("jkooa", C.c_int32),
                ("dxk", C.c_float), ("dyk", C.c_float), ("ahmin", C.c_float), ("met", C.POINTER(GralMet))]


PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f4"), ("ahint", "<f4"), ("i", "<i4"), ("j", "<i4")])


class GralStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("iteration_loops", C.c_int32),
        ("converged", C.c_int32), ("convergence_problem", C.c_int32),
        ("delta_first", C.c_double), ("delta_finish", C.c_double),
        ("n_history", C.c_int32), ("delta_history", C.c_double * MAX_HISTORY),
        ("uk_unrealistic", C.c_int32), ("vk_unrealistic", C.c_int32),
        ("wk_unrealistic", C.c_int32),
        ("geschw_max", C.c_double), ("topwind", C.c_float), ("dtime", C.c_float),
        ("frund", C.c_double), ("last_delta_umax", C.c_float),
        ("trace_delta_umax", _fp), ("trace_capacity", C.c_int32),
        ("ms_total", C.c_double), ("ms_upload", C.c_double),
        ("ms_iterate", C.c_double), ("ms_download", C.c_double),
        ("layout", C.c_int32), ("launch_variant", C.c_int32),
        ("launches_per_iteration", C.c_int32),
    ]


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays passed through the ABI must be C-contiguous")
    return a.ctypes.data_as(C.POINTER(ctype))



class GralVjpStats(C.Structure):
    """gral_vjp_stats: device times of the adjoint's forward run, recomputation and reverse sweeps."""
    _fields_ = [("iterations", C.c_int32), ("checkpoint_every", C.c_int32),
                ("ms_forward", C.c_double), ("ms_recompute", C.c_double), ("ms_reverse", C.c_double),
                ("ms_total", C.c_double)]

@dataclass
class StaticArrays:
    """Per-grid inputs (``gral_static``) as numpy arrays with the reference's index ranges."""
    kkart: np.ndarray            # int16 [NII+2, NJJ+2]
    advdom: np.ndarray           # uint8 [NII+2, NJJ+2]
    cutk: np.ndarray             # float32 [NII+2, NJJ+2]
    cov: np.ndarray              # float32 [NII+2, NJJ+2]
    z0: np.ndarray               # float32 [NII+2, NJJ+2]
    z0_init: np.ndarray          # float32 [NII+2, NJJ+2]
    ob_init: np.ndarray          # float32 [NII+2, NJJ+2]
    ust_init: np.ndarray         # float32 [NII+2, NJJ+2]
    dzk: np.ndarray              # float32 [NKK+2]
    hokart: np.ndarray           # float32 [NKK+2]
    veg: Optional[np.ndarray] = None       # float32 [NII+2, NJJ+2, NKK+2]
    veg_mask: Optional[np.ndarray] = None  # uint8 [NII+2, NJJ+2]

    def to_c(self) -> GralStatic:
        return GralStatic(
            kkart=_ptr(self.kkart, C.c_int16), advdom=_ptr(self.advdom, C.c_uint8),
            cutk=_ptr(self.cutk, C.c_float), cov=_ptr(self.cov, C.c_float),
            z0=_ptr(self.z0, C.c_float), z0_init=_ptr(self.z0_init, C.c_float),
            ob_init=_ptr(self.ob_init, C.c_float), ust_init=_ptr(self.ust_init, C.c_float),
            veg=_ptr(self.veg, C.c_float), veg_mask=_ptr(self.veg_mask, C.c_uint8),
            dzk=_ptr(self.dzk, C.c_float), hokart=_ptr(self.hokart, C.c_float))


@dataclass
class FieldArrays:
    """Per-situation fields (``gral_fields``), float32 [NII+2, NJJ+2, NKK+2], k fastest."""
    uk: np.ndarray
    vk: np.ndarray
    wk: np.ndarray
    turb: Optional[np.ndarray] = None
    tdiss: Optional[np.ndarray] = None

    def copy(self) -> "FieldArrays":
        c = lambda a: None if a is None else a.copy()
        return FieldArrays(self.uk.copy(), self.vk.copy(), self.wk.copy(), c(self.turb), c(self.tdiss))

    def to_c(self) -> GralFields:
        return GralFields(uk=_ptr(self.uk, C.c_float), vk=_ptr(self.vk, C.c_float),
                          wk=_ptr(self.wk, C.c_float), turb=_ptr(self.turb, C.c_float),
                          tdiss=_ptr(self.tdiss, C.c_float))


def params_to_c(p: dict) -> GralParams:
    out = GralParams()
    for name, _ in GralParams._fields_:
        if name not in p:
            raise KeyError(f"missing solver parameter {name!r}")
        setattr(out, name, p[name])
    return out


def stats_to_dict(s: GralStats) -> dict:
    d = {name: getattr(s, name) for name, _ in GralStats._fields_
         if name not in ("delta_history", "trace_delta_umax")}
    d["delta_history"] = [s.delta_history[i] for i in range(min(s.n_history, MAX_HISTORY))]
    return d


@dataclass
class MetProfile:
    """Met input of one situation (``gral_met``): heights, wind components at them (index 0
    unused, as in the reference's arrays), the profile's Obukhov length and optionally one per
    column (adaptive roughness)."""
    heights: np.ndarray
    obs_u: np.ndarray
    obs_v: np.ndarray
    ob_length: float
    ol_column: Optional[np.ndarray] = None

    def to_c(self) -> GralMet:
        self._keep = [np.ascontiguousarray(a, dtype=np.float32) for a in (self.heights, self.obs_u, self.obs_v)]
        self._ol = None if self.ol_column is None else np.ascontiguousarray(self.ol_column, dtype=np.float32)
        h, u, v = self._keep
        return GralMet(n_heights=h.size - 1, measurement_height=_ptr(h, C.c_float), obs_u=_ptr(u, C.c_float),
                       obs_v=_ptr(v, C.c_float), ob_length=float(self.ob_length),
                       ol_column=_ptr(self._ol, C.c_float))


def veg_points_to_c(points) -> "C.Array":
    """``gral_veg_point`` array from dicts with crown_height, trunk_height, trunk_lad, crown_lad,
    cov, i, j and drag."""
    arr = (GralVegPoint * max(len(points), 1))()
    for q, p in enumerate(points):
        arr[q] = GralVegPoint(p["crown_height"], p["trunk_height"], p["trunk_lad"], p["crown_lad"], p["cov"],
                              p["i"], p["j"], int(p.get("drag", 1)), 0)
    return arr

