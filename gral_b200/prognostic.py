"""Host-side mirror of ``PrognosticFlowfield.Calculate()`` over the C ABI of ``libgralprog.so``.

``PrognosticSolver.calculate`` is the drop-in for one weather situation: it reads the fields,
runs the SIMPLE loop on the GPU and writes UK/VK/WK (and TURB/TDISS) back in place, like the
reference's static method does with ``Program.UK/VK/WK`` (PrognosticFlowfield.cs:32).
``calculate_batch`` solves many situations of one grid together.  There is no CPU fallback:
a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import build as _build
from .abi import (GRAL_OK, PARTICLE_DTYPE, STATUS_NAMES, FieldArrays, GralFields, GralFlatGrid, GralMet,
                  GralParams, GralStatic, GralStats, GralVegPoint, GralVjpStats, GralWindGrid, MetProfile,
                  StaticArrays, params_to_c, stats_to_dict, veg_points_to_c)

_lib = None

EXPORTS = ["gral_prog_version", "gral_prog_create", "gral_prog_solve", "gral_prog_solve_batch",
           "gral_prog_load", "gral_prog_iterate", "gral_prog_iterate_timed", "gral_prog_store",
           "gral_prog_last_error", "gral_prog_destroy", "gral_prog_check_speeds_noalloc",
           "gral_prog_gff_size", "gral_prog_gff_pack", "gral_prog_gff_pack_timed", "gral_prog_gff_unpack",
           "gral_prog_subdomains", "gral_prog_flat_init", "gral_prog_vegetation", "gral_prog_prep_last_ms",
           "gral_prog_wind_at", "gral_prog_solve_instances", "gral_prog_solve_batch_devices", "gral_prog_load_flat", "gral_prog_vjp_forward",
           "gral_prog_vjp"]

# payload modes of gral_prog_gff_pack (GFFWrite.cs writingMode 0, 1, 2 and the model-2 .tke file)
GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN, GFF_TKE = 0, 1, 2, 3
GFF_HEADER_BYTES = 32

PHASES = ["bc", "pressure", "velcorr", "average", "u", "v", "w", "tke", "bookkeeping", "pvau"]


class GralError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def lib(build_if_stale: bool = True):
    """Load libgralprog.so (building it first when the sources are newer and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_stale and _build.stale():
        try:
            _build.build()
        except RuntimeError:
            if not os.path.exists(path):
                raise
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing; run `python -m gral_b200.build`")
    L = C.CDLL(path)
    L.gral_prog_version.restype = C.c_int
    L.gral_prog_create.argtypes = [C.c_int32] * 5 + [C.POINTER(C.c_void_p)]
    L.gral_prog_create.restype = C.c_int
    L.gral_prog_solve.argtypes = [C.c_void_p, C.POINTER(GralParams), C.POINTER(GralStatic),
                                  C.POINTER(GralFields), C.POINTER(GralStats)]
    L.gral_prog_solve.restype = C.c_int
    L.gral_prog_solve_batch.argtypes = [C.c_void_p, C.c_int32, C.POINTER(GralParams), C.POINTER(GralStatic),
                                        C.POINTER(GralFields), C.POINTER(GralStats)]
    L.gral_prog_solve_batch.restype = C.c_int
    L.gral_prog_load.argtypes = [C.c_void_p, C.c_int32, C.POINTER(GralParams), C.POINTER(GralStatic),
                                 C.POINTER(GralFields)]
    L.gral_prog_load.restype = C.c_int
    L.gral_prog_iterate.argtypes = [C.c_void_p]
    L.gral_prog_iterate.restype = C.c_int
    L.gral_prog_iterate_timed.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.gral_prog_iterate_timed.restype = C.c_int
    L.gral_prog_store.argtypes = [C.c_void_p, C.POINTER(GralFields), C.POINTER(GralStats)]
    L.gral_prog_store.restype = C.c_int
    L.gral_prog_last_error.argtypes = [C.c_void_p]
    L.gral_prog_last_error.restype = C.c_char_p
    L.gral_prog_destroy.argtypes = [C.c_void_p]
    L.gral_prog_destroy.restype = None
    L.gral_prog_check_speeds_noalloc.argtypes = [C.c_int32] * 4 + [C.c_double] + [C.c_void_p] * 5 + \
        [C.POINTER(C.c_int32), C.c_void_p]
    L.gral_prog_check_speeds_noalloc.restype = C.c_int
    L.gral_prog_gff_size.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_uint64)]
    L.gral_prog_gff_size.restype = C.c_int
    L.gral_prog_gff_pack.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int32,
                                     C.c_void_p, C.c_uint64]
    L.gral_prog_gff_pack.restype = C.c_int
    L.gral_prog_gff_pack_timed.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    L.gral_prog_gff_pack_timed.restype = C.c_int
    L.gral_prog_gff_unpack.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32)]
    L.gral_prog_gff_unpack.restype = C.c_int
    vp = C.c_void_p
    L.gral_prog_subdomains.argtypes = [vp, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int32, vp, vp]
    L.gral_prog_subdomains.restype = C.c_int
    L.gral_prog_flat_init.argtypes = [vp, C.POINTER(GralFlatGrid), vp, vp, vp, vp, C.POINTER(GralMet), vp, vp,
                                      C.POINTER(C.c_int32), C.POINTER(GralFields)]
    L.gral_prog_flat_init.restype = C.c_int
    L.gral_prog_vegetation.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_int32,
                                       C.POINTER(GralVegPoint), vp, vp, vp]
    L.gral_prog_vegetation.restype = C.c_int
    L.gral_prog_prep_last_ms.argtypes = [vp, C.POINTER(C.c_double)]
    L.gral_prog_prep_last_ms.restype = C.c_int
    L.gral_prog_wind_at.argtypes = [vp, C.c_int32, C.POINTER(GralWindGrid), vp, vp, C.c_int32, vp, vp, vp, vp, vp]
    L.gral_prog_wind_at.restype = C.c_int
    L.gral_prog_solve_instances.argtypes = [C.c_int32, C.POINTER(GralParams), C.POINTER(GralStatic),
                                            C.POINTER(GralFields), C.POINTER(GralStats), C.POINTER(C.c_int32),
                                            C.c_int32, C.c_uint64]
    L.gral_prog_solve_instances.restype = C.c_int
    L.gral_prog_solve_batch_devices.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(GralParams),
                                                C.POINTER(GralStatic), C.POINTER(GralFields), C.POINTER(GralStats)]
    L.gral_prog_solve_batch_devices.restype = C.c_int
    L.gral_prog_load_flat.argtypes = [vp, C.c_int32, C.POINTER(GralParams), C.POINTER(GralStatic), C.POINTER(GralMet),
                                      C.POINTER(GralFlatGrid), C.POINTER(GralFields)]
    L.gral_prog_load_flat.restype = C.c_int
    L.gral_prog_vjp_forward.argtypes = [vp, C.POINTER(GralParams), C.POINTER(GralStatic), C.POINTER(GralFields),
                                        C.c_int32, C.c_int32]
    L.gral_prog_vjp_forward.restype = C.c_int
    L.gral_prog_vjp.argtypes = [vp] + [vp] * 7 + [C.POINTER(GralVjpStats)]
    L.gral_prog_vjp.restype = C.c_int
    _lib = L
    return L


class PrognosticSolver:
    """A solver context for grids up to (nii, njj, nkk, kadvmax) and up to max_batch situations."""

    def __init__(self, nii: int, njj: int, nkk: int, kadvmax: int, max_batch: int = 1):
        self._L = lib()
        self._ctx = C.c_void_p()
        rc = self._L.gral_prog_create(nii, njj, nkk, kadvmax, max_batch, C.byref(self._ctx))
        if rc != GRAL_OK:
            raise GralError(rc, "gral_prog_create failed")
        self._keep: list = []

    def _check(self, rc: int):
        if rc != GRAL_OK:
            msg = self._L.gral_prog_last_error(self._ctx).decode()
            raise GralError(rc, msg)

    def close(self):
        if self._ctx:
            self._L.gral_prog_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stats_array(n: int, traces: Optional[Sequence[np.ndarray]]):
        st = (GralStats * n)()
        if traces is not None:
            for b, t in enumerate(traces):
                st[b].trace_delta_umax = t.ctypes.data_as(C.POINTER(C.c_float))
                st[b].trace_capacity = t.size
        return st

    def calculate(self, params: dict, static: StaticArrays, fields: FieldArrays,
                  trace: Optional[np.ndarray] = None) -> dict:
        """One situation, in place on ``fields``; returns the run statistics."""
        return self.calculate_batch([params], static, [fields], None if trace is None else [trace])[0]

    def calculate_batch(self, params: Sequence[dict], static: StaticArrays, fields: Sequence[FieldArrays],
                        traces: Optional[Sequence[np.ndarray]] = None) -> List[dict]:
        n = len(params)
        pa = (GralParams * n)(*[params_to_c(p) for p in params])
        s = static.to_c()
        fa = (GralFields * n)(*[f.to_c() for f in fields])
        st = self._stats_array(n, traces)
        self._check(self._L.gral_prog_solve_batch(self._ctx, n, pa, C.byref(s), fa, st))
        return [stats_to_dict(st[b]) for b in range(n)]

    # split form: inputs resident on the device between load and store
    def load(self, params: Sequence[dict], static: StaticArrays, fields: Sequence[FieldArrays]):
        n = len(params)
        pa = (GralParams * n)(*[params_to_c(p) for p in params])
        s = static.to_c()
        fa = (GralFields * n)(*[f.to_c() for f in fields])
        self._keep = [pa, s, fa, static, fields]
        self._check(self._L.gral_prog_load(self._ctx, n, pa, C.byref(s), fa))

    def load_flat(self, params: Sequence[dict], static: StaticArrays, mets: Sequence[MetProfile], grid: dict,
                  fields: Sequence[FieldArrays]):
        """Split-form load whose initial U, V, W are built on the device from each situation's met
        profile (flat-terrain set-up); ``fields`` receive the results at ``store``."""
        n = len(params)
        pa = (GralParams * n)(*[params_to_c(p) for p in params])
        s = static.to_c()
        ma = (GralMet * n)(*[m.to_c() for m in mets])
        g = GralFlatGrid(**grid)
        fa = (GralFields * n)(*[f.to_c() for f in fields])
        self._keep = [pa, s, ma, g, fa, static, fields, mets]
        self._check(self._L.gral_prog_load_flat(self._ctx, n, pa, C.byref(s), ma, C.byref(g), fa))

    def iterate(self):
        self._check(self._L.gral_prog_iterate(self._ctx))

    def iterate_timed(self, iterations: int):
        """Run exactly `iterations` SIMPLE iterations; returns (total_ms, {phase: summed ms})."""
        ph = (C.c_double * len(PHASES))()
        tot = C.c_double()
        self._check(self._L.gral_prog_iterate_timed(self._ctx, iterations, ph, C.byref(tot)))
        return tot.value, {name: ph[q] for q, name in enumerate(PHASES)}

    def store(self, fields: Sequence[FieldArrays], traces=None) -> List[dict]:
        n = len(fields)
        fa = (GralFields * n)(*[f.to_c() for f in fields])
        st = self._stats_array(n, traces)
        self._check(self._L.gral_prog_store(self._ctx, fa, st))
        return [stats_to_dict(st[b]) for b in range(n)]

    # discrete adjoint of the unrolled SIMPLE iterations (model 1, parity width 8, no rounding)
    def vjp_forward(self, params: dict, static: StaticArrays, fields: FieldArrays, iterations: int,
                    checkpoint_every: int = 20):
        """Forward run of the differentiated map: `iterations` SIMPLE iterations of one situation,
        in place on ``fields``, with checkpoints kept on the device for ``vjp``."""
        p = params_to_c(params)
        s = static.to_c()
        f = fields.to_c()
        self._keep = [p, s, f, static, fields]
        self._check(self._L.gral_prog_vjp_forward(self._ctx, C.byref(p), C.byref(s), C.byref(f), iterations,
                                                  checkpoint_every))

    def vjp(self, dj_duk: Optional[np.ndarray], dj_dvk: Optional[np.ndarray] = None,
            dj_dwk: Optional[np.ndarray] = None):
        """Vector-Jacobian product of the last ``vjp_forward``: cotangents of its final UK, VK, WK
        (float32 host layout, None = zero) -> (dJ/dVEG, dJ/dUK0, dJ/dVK0, dJ/dWK0, stats dict)."""
        ref = next(a for a in (dj_duk, dj_dvk, dj_dwk) if a is not None)
        shape = ref.shape
        ins = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (dj_duk, dj_dvk, dj_dwk)]
        outs = [np.zeros(shape, np.float32) for _ in range(4)]
        st = GralVjpStats()
        ptr = [None if a is None else a.ctypes.data for a in ins]
        self._check(self._L.gral_prog_vjp(self._ctx, *ptr, *(o.ctypes.data for o in outs), C.byref(st)))
        stats = {name: getattr(st, name) for name, _ in GralVjpStats._fields_}
        return outs[0], outs[1], outs[2], outs[3], stats

    # flow-field cache payloads (GFFWrite.cs / GFFRead.cs); the zip container stays with the caller
    def gff_size(self, mode: int) -> int:
        n = C.c_uint64()
        self._check(self._L.gral_prog_gff_size(self._ctx, mode, C.byref(n)))
        return n.value

    def gff_pack(self, situation: int, mode: int, wind_dir: float = 0.0, wind_speed: float = 0.0,
                 stability_class: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Payload bytes (header + data) of one situation of the last store, packed on the GPU."""
        n = self.gff_size(mode)
        if out is None:
            out = np.empty(n, np.uint8)
        self._check(self._L.gral_prog_gff_pack(self._ctx, situation, mode, wind_dir, wind_speed, stability_class,
                                               out.ctypes.data, out.nbytes))
        return out[:n]

    # flow-field set-up before the solve (ReadGeometryAndDomains.cs, MicroscaleFlat.cs, ReadVegetation.cs)
    def subdomains(self, cutk: np.ndarray, nii: int, njj: int, dxk: float, dyk: float, factor: int = 15) -> np.ndarray:
        """ADVDOM [NII+2][NJJ+2] of the prognostic sub-domains around the buildings."""
        cutk = np.ascontiguousarray(cutk, np.float32)
        adv = np.zeros((nii + 2, njj + 2), np.uint8)
        self._check(self._L.gral_prog_subdomains(self._ctx, nii, njj, dxk, dyk, factor, cutk.ctypes.data,
                                                 adv.ctypes.data))
        return adv

    def flat_init(self, grid: dict, cutk: np.ndarray, dzk: np.ndarray, hokart: np.ndarray, met: MetProfile,
                  advdom: Optional[np.ndarray] = None):
        """Flat-terrain set-up of one situation; returns (kkart, ahk, kadvmax, FieldArrays)."""
        nii, njj, nkk = grid["nii"], grid["njj"], grid["nkk"]
        g = GralFlatGrid(**grid)
        cutk, dzk, hokart = (np.ascontiguousarray(a, np.float32) for a in (cutk, dzk, hokart))
        adv = None if advdom is None else np.ascontiguousarray(advdom, np.uint8)
        shape = (nii + 2, njj + 2, nkk + 2)
        f = FieldArrays(*(np.empty(shape, np.float32) for _ in range(3)))
        kk = np.empty((nii + 2, njj + 2), np.int16)
        ahk = np.empty((nii + 2, njj + 2), np.float32)
        kadv = C.c_int32()
        m = met.to_c()
        fc = f.to_c()
        self._check(self._L.gral_prog_flat_init(self._ctx, C.byref(g), cutk.ctypes.data, dzk.ctypes.data,
                                                hokart.ctypes.data, None if adv is None else adv.ctypes.data,
                                                C.byref(m), kk.ctypes.data, ahk.ctypes.data, C.byref(kadv),
                                                C.byref(fc)))
        return kk, ahk, kadv.value, f

    def vegetation(self, nii: int, njj: int, nkk: int, kkart: np.ndarray, dzk: np.ndarray, hokart: np.ndarray,
                   points: Sequence[dict], cov: np.ndarray):
        """VEG [NII+2][NJJ+2][NKK+2], its mask and COV after rasterising the vegetation lines."""
        kk = np.ascontiguousarray(kkart, np.int16)
        dz, ho = (np.ascontiguousarray(a, np.float32) for a in (dzk, hokart))
        cov = np.array(cov, dtype=np.float32, copy=True, order="C")
        veg = np.empty((nii + 2, njj + 2, nkk + 2), np.float32)
        mask = np.empty((nii + 2, njj + 2), np.uint8)
        pts = veg_points_to_c(points)
        self._check(self._L.gral_prog_vegetation(self._ctx, nii, njj, nkk, kk.ctypes.data, dz.ctypes.data,
                                                 ho.ctypes.data, len(points), pts, veg.ctypes.data,
                                                 mask.ctypes.data, cov.ctypes.data))
        return veg, mask, cov

    def wind_at(self, situation: int, grid: dict, dzk: Optional[np.ndarray], hokart: Optional[np.ndarray],
                particles: np.ndarray, met: Optional[MetProfile] = None):
        """U, V, W and IndexK at particle positions (``PARTICLE_DTYPE`` records), interpolated from
        the stored fields of `situation` as Zeitschleife.IntWindCalculate does."""
        p = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        n = p.size
        ux, uy, uz = (np.empty(n, np.float32) for _ in range(3))
        kk = np.empty(n, np.int32)
        m = None if met is None else met.to_c()
        g = GralWindGrid(grid.get("terrain", 0), grid.get("buildings", 1), grid.get("ikooa", 0), grid.get("jkooa", 0),
                         grid["dxk"], grid["dyk"], grid.get("ahmin", 0.0),
                         C.pointer(m) if m is not None else C.POINTER(GralMet)())
        dz = None if dzk is None else np.ascontiguousarray(dzk, np.float32)
        ho = None if hokart is None else np.ascontiguousarray(hokart, np.float32)
        self._check(self._L.gral_prog_wind_at(self._ctx, situation, C.byref(g),
                                              None if dz is None else dz.ctypes.data,
                                              None if ho is None else ho.ctypes.data, n, p.ctypes.data,
                                              ux.ctypes.data, uy.ctypes.data, uz.ctypes.data, kk.ctypes.data))
        return ux, uy, uz, kk

    def prep_last_ms(self) -> float:
        """Device ms of the kernels of the last subdomains/flat_init/vegetation call."""
        ms = C.c_double()
        self._check(self._L.gral_prog_prep_last_ms(self._ctx, C.byref(ms)))
        return ms.value

    def gff_pack_timed(self, situation: int, mode: int, repeats: int) -> float:
        """Mean device ms of one pack launch (L2 flushed before each), no copy to the host."""
        ms = C.c_double()
        self._check(self._L.gral_prog_gff_pack_timed(self._ctx, situation, mode, repeats, C.byref(ms)))
        return ms.value

    def gff_unpack(self, payload, nii: int, njj: int, nkk: int, dxk: float,
                   kkart: Optional[np.ndarray] = None, out: Optional[FieldArrays] = None):
        """Read a flow-field payload on the GPU into flat [NII+2][NJJ+2][NKK+2] arrays.

        Returns ``(uk, vk, wk, (wind_dir, wind_speed, stability_class, flag))``; with a format flag
        the reference's reader skips (not -1, -2, -3) the arrays come back untouched.
        """
        buf = payload if isinstance(payload, np.ndarray) else np.frombuffer(bytes(payload), np.uint8)
        buf = np.ascontiguousarray(buf, np.uint8)
        shape = (nii + 2, njj + 2, nkk + 2)
        if out is None:
            uk, vk, wk = (np.zeros(shape, np.float32) for _ in range(3))
        else:
            uk, vk, wk = out.uk, out.vk, out.wk
        kk = None if kkart is None else np.ascontiguousarray(kkart, np.int16)
        d, v, st, fl = C.c_float(), C.c_float(), C.c_int32(), C.c_int32()
        self._check(self._L.gral_prog_gff_unpack(self._ctx, buf.ctypes.data, buf.nbytes, nii, njj, nkk, dxk,
                                                 None if kk is None else kk.ctypes.data, uk.ctypes.data,
                                                 vk.ctypes.data, wk.ctypes.data, C.byref(d), C.byref(v),
                                                 C.byref(st), C.byref(fl)))
        return uk, vk, wk, (d.value, v.value, st.value, fl.value)


def check_speeds_noalloc(nii: int, njj: int, nkk: int, vert_cells_ff: int, geschw_max: float,
                         uk_ptr: int, vk_ptr: int, wk_ptr: int, advdom_ptr: int, kkart_ptr: int,
                         stream: int = 0) -> tuple:
    """Unrealistic-wind-speed counts (U, V, W, non-finite) of a flow field that is already on the
    GPU, without any device allocation (``gral_prog_check_speeds_noalloc``).

    For callers that hold the solved field in device memory and cannot allocate there: one whose
    device memory is committed to its own pool, or that must not let cudaMalloc/cudaFree
    synchronise the device while other streams run.  The pointers are device addresses of
    [NII+2][NJJ+2][NKK+2] float32 (U, V, W), uint8 ADVDOM and int16 KKART arrays
    ([NII+2][NJJ+2]); ``stream`` is a cudaStream_t handle (0: the legacy default stream).  Grids
    with more than ``GRAL_NOALLOC_MAX_ROWS`` (4096) rows are rejected; concurrent calls on one
    device race on the shared fixed scratch and must be serialised.
    """
    L = lib()
    out = (C.c_int32 * 4)()
    rc = L.gral_prog_check_speeds_noalloc(nii, njj, nkk, vert_cells_ff, float(geschw_max), uk_ptr, vk_ptr,
                                          wk_ptr, advdom_ptr, kkart_ptr, out, stream)
    if rc != GRAL_OK:
        raise GralError(rc, "gral_prog_check_speeds_noalloc failed")
    return tuple(int(x) for x in out)


def solve_instances(params: Sequence[dict], statics: Sequence[StaticArrays], fields: Sequence[FieldArrays],
                    max_concurrent: int = 8, hbm_bytes: int = 0):
    """Independent situations on grids of different sizes, several at once on one GPU
    (``gral_prog_solve_instances``); fields are updated in place.  Returns (stats, status, rc)."""
    L = lib()
    n = len(params)
    pa = (GralParams * n)(*[params_to_c(p) for p in params])
    sa = (GralStatic * n)(*[st.to_c() for st in statics])
    fa = (GralFields * n)(*[f.to_c() for f in fields])
    st = (GralStats * n)()
    status = (C.c_int32 * n)()
    rc = L.gral_prog_solve_instances(n, pa, sa, fa, st, status, max_concurrent, hbm_bytes)
    stats = [stats_to_dict(st[b]) for b in range(n)]
    return stats, [int(x) for x in status], rc


def solve_batch_devices(devices: Sequence[int], params: Sequence[dict], static: StaticArrays,
                        fields: Sequence[FieldArrays]):
    """A batch of situations on one grid spread over several GPUs of the node
    (``gral_prog_solve_batch_devices``): devices[d] takes the d-th contiguous shard; fields are
    updated in place.  Returns (stats, rc)."""
    L = lib()
    n, nd = len(params), len(devices)
    dv = (C.c_int32 * max(nd, 1))(*devices)
    pa = (GralParams * n)(*[params_to_c(p) for p in params])
    sa = static.to_c()
    fa = (GralFields * n)(*[f.to_c() for f in fields])
    st = (GralStats * n)()
    rc = L.gral_prog_solve_batch_devices(nd, dv, n, pa, C.byref(sa), fa, st)
    return [stats_to_dict(st[b]) for b in range(n)], rc

