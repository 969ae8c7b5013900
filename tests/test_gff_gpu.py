"""GPU parity of the flow-field cache payloads: device pack/unpack against ``oracle/gff.py``.

``gral_prog_gff_pack`` converts the fields resident on the device after a store into the .gff
formats (flags -1, -2, -3) and the model-2 .tke file; its bytes must equal the CPU restatement's
for the same fields (the fields ``gral_prog_store`` returned), including values that clamp, NaN
and half-way roundings placed above the solved sub-domain, every situation of a batch, and the
fields after the diagnostic step.  ``gral_prog_gff_unpack`` must give exactly the arrays the
CPU reader gives, and reject the files the reference's reader rejects.
"""
import struct

import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.prognostic import (GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN, GFF_TKE, GralError,
                                  PrognosticSolver)
from oracle import gff as O

pytestmark = pytest.mark.gpu

HDR = dict(wind_dir=247.5, wind_speed=3.5, stab=4)


def plant(dom, f, model):
    """Values the conversions treat specially, at the top levels, which the solve leaves alone."""
    n = dom.nkk
    f.uk[3, 4, n] = 400.0            # clamps to 32767
    f.vk[5, 2, n] = -400.0           # clamps to -32768
    f.wk[6, 7, n + 1] = np.nan       # converts to 0
    f.uk[7, 3, n] = np.float32(0.125)    # 12.5: half-way for the terrain format's rounding
    f.vk[8, 5, n] = np.float32(-0.375)
    if model == 2:
        f.turb[4, 4, n] = np.float32(0.125)
        f.turb[2, 6, n] = 1000.0


def turb_from_presolve(dom, s, ps, fs):
    """Model 2 initialises TURB/TDISS over the whole column (turb_init 0); a first solve gives
    fields that a second load takes as they are (turb_init 1), so values planted in TURB stay."""
    s.load(ps, dom.static, fs)
    s.iterate()
    s.store(fs)
    for p in ps:
        p["turb_init"] = 1


def solved(model, sits, post_diagnostic=0, special=True, turb_nan=False):
    dom = prep.small_domain(16, 14, seed=31)
    ps = [dom.params(x, model=model, iterations=4, post_diagnostic=post_diagnostic) for x in sits]
    fs = [prep.initial_fields(dom, x, model) for x in sits]
    s = PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(sits))
    if model == 2 and (special or turb_nan):
        turb_from_presolve(dom, s, ps, fs)
    if special:
        for f in fs:
            plant(dom, f, model)
    if turb_nan:
        fs[0].turb[3, 3, dom.nkk] = np.nan
    s.load(ps, dom.static, fs)
    s.iterate()
    s.store(fs)
    return dom, s, fs


def oracle_pack(mode, dom, f):
    return O.pack(mode, f.uk, f.vk, f.wk, kkart=dom.static.kkart, turb=f.turb, dxk=dom.dxk, **HDR)


def gpu_pack(s, b, mode):
    return s.gff_pack(b, mode, HDR["wind_dir"], HDR["wind_speed"], HDR["stab"]).tobytes()


@pytest.mark.parametrize("model", [1, 2])
def test_pack_matches_oracle(gpu_required, model):
    sits = [prep.Situation(direction_deg=230.0), prep.Situation(direction_deg=95.0, speed_10m=4.0)]
    dom, s, fs = solved(model, sits)
    with s:
        modes = [GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN] + ([GFF_TKE] if model == 2 else [])
        for b in range(len(sits)):
            for mode in modes:
                want = oracle_pack(mode, dom, fs[b])
                assert s.gff_size(mode) == len(want)
                got = gpu_pack(s, b, mode)
                assert got == want, (model, b, mode)
        # the planted values reached the payload: clamped, NaN -> 0, half-even rounding
        d = np.frombuffer(oracle_pack(GFF_COLUMNS, dom, fs[0]), "<i2", offset=32).reshape(
            dom.nii + 1, dom.njj + 1, dom.nkk + 1, 3)
        assert d[2, 3, dom.nkk, 0] == 32767 and d[4, 1, dom.nkk, 1] == -32768 and d[5, 6, dom.nkk, 2] == 0
        if model == 2:
            t = np.frombuffer(oracle_pack(GFF_TKE, dom, fs[0]), "<i2", offset=32).reshape(dom.nii, dom.njj, dom.nkk)
            assert t[3, 3, dom.nkk - 1] == 12 and t[1, 5, dom.nkk - 1] == 32767


def test_pack_after_diagnostic(gpu_required):
    sits = [prep.Situation(direction_deg=200.0)]
    dom, s, fs = solved(1, sits, post_diagnostic=1, special=False)
    with s:
        for mode in (GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN):
            assert gpu_pack(s, 0, mode) == oracle_pack(mode, dom, fs[0])


@pytest.mark.parametrize("mode", [GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN])
def test_unpack_matches_oracle(gpu_required, mode):
    dom = prep.small_domain(16, 14, seed=5)
    rng = np.random.default_rng(mode)
    shape = (dom.nii + 2, dom.njj + 2, dom.nkk + 2)
    U, V, W = ((rng.standard_normal(shape) * 40).astype(np.float32) for _ in range(3))
    payload = O.pack(mode, U, V, W, kkart=dom.static.kkart, dxk=dom.dxk, **HDR)
    want = O.unpack(payload, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for _ in range(2):       # a second call reuses the buffers and must give the same arrays
            got = s.gff_unpack(payload, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart)
            for a, b in zip(got[:3], want[:3]):
                np.testing.assert_array_equal(a, b)
            assert got[3] == (np.float32(247.5), np.float32(3.5), 4, -1 - mode)


def test_errors(gpu_required):
    sits = [prep.Situation()]
    dom = prep.small_domain(16, 14, seed=31)
    p = [dom.params(sits[0], model=1, iterations=2)]
    f = [prep.initial_fields(dom, sits[0], 1)]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        s.load(p, dom.static, f)
        with pytest.raises(GralError) as e:
            s.gff_pack(0, GFF_COLUMNS)
        assert e.value.code == abi.GRAL_ESTATE                 # nothing stored yet
        s.iterate()
        s.store(f)
        with pytest.raises(GralError) as e:
            s.gff_pack(0, GFF_TKE)
        assert e.value.code == abi.GRAL_EINVAL                 # no TKE field in model 1
        with pytest.raises(GralError) as e:
            s.gff_pack(1, GFF_COLUMNS)
        assert e.value.code == abi.GRAL_EINVAL                 # situation out of range
        with pytest.raises(GralError) as e:
            s.gff_pack(0, GFF_COLUMNS, out=np.empty(s.gff_size(GFF_COLUMNS) - 1, np.uint8))
        assert e.value.code == abi.GRAL_EINVAL                 # buffer too small
        good = gpu_pack(s, 0, GFF_TERRAIN)
        kk = dom.static.kkart
        bad_cases = [
            (good, dom.nii, dom.njj, dom.nkk + 1, dom.dxk, kk),
            (good, dom.nii, dom.njj + 1, dom.nkk, dom.dxk, kk),
            (good, dom.nii - 1, dom.njj, dom.nkk, dom.dxk, kk),
            (good, dom.nii, dom.njj, dom.nkk, dom.dxk * 2, kk),
            (good[:-2], dom.nii, dom.njj, dom.nkk, dom.dxk, kk),
            (good, dom.nii, dom.njj, dom.nkk, dom.dxk, np.where(kk == kk[5, 5], kk + 1, kk).astype(np.int16)),
            (good, dom.nii, dom.njj, dom.nkk, dom.dxk, None),
        ]
        for args in bad_cases:
            with pytest.raises(GralError) as e:
                s.gff_unpack(*args)
            assert e.value.code == abi.GRAL_EINVAL
        # an unknown format flag: the reference's reader stops there and succeeds
        odd = good[:28] + struct.pack("<i", -9) + good[32:]
        keep = abi.FieldArrays(*(np.full((dom.nii + 2, dom.njj + 2, dom.nkk + 2), 7.0, np.float32)
                                  for _ in range(3)))
        u, v, w, info = s.gff_unpack(odd, dom.nii, dom.njj, dom.nkk, dom.dxk, out=keep)
        assert info[3] == -9 and np.all(u == 7.0) and np.all(w == 7.0)
        # and the context still works
        assert gpu_pack(s, 0, GFF_LEVELS) == oracle_pack(GFF_LEVELS, dom, f[0])


def test_tke_nonfinite(gpu_required):
    dom, s, f = solved(2, [prep.Situation()], special=False, turb_nan=True)
    assert np.isnan(f[0].turb[3, 3, dom.nkk])
    with s:
        with pytest.raises(GralError) as e:
            s.gff_pack(0, GFF_TKE)
        assert e.value.code == abi.GRAL_ENONFINITE
        assert gpu_pack(s, 0, GFF_COLUMNS) == oracle_pack(GFF_COLUMNS, dom, f[0])


def test_full_size_round_trip(gpu_required):
    """The 400x400 production grid: every format byte-exact, and read back exactly."""
    dom = prep.city_domain()
    sit = prep.Situation(direction_deg=225.0, speed_10m=2.0, z0=0.5)
    f = prep.initial_fields(dom, sit)
    plant(dom, f, 1)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        s.load([dom.params(sit, iterations=1)], dom.static, [f])
        s.store([f])
        for mode in (GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN):
            got = gpu_pack(s, 0, mode)
            assert got == oracle_pack(mode, dom, f), mode
            back = s.gff_unpack(got, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart)
            want = O.unpack(got, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart)
            for a, b in zip(back[:3], want[:3]):
                np.testing.assert_array_equal(a, b)
