"""The CPU restatement of the flow-field set-up (``oracle/prep.cpp``) on known answers.

The reference holds no fixtures for these routines, so the restatement is checked against
values derived by hand from the reference's rules: sub-domain rectangles for a single building
cell, the initial profile (power law with the stable and unstable exponents, interpolation
between three heights, calling the C library's powf as .NET's MathF.Pow does), the obstacle and
edge rules of the initial field, KKART/AHK/KADVMAX, one near-wall damping factor, and the
vegetation crown/trunk rule with a later line overriding an earlier one in the same cell.
"""
import ctypes
import ctypes.util
import math

import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.abi import MetProfile
from oracle import prep as OP

F32 = np.float32
_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.powf.restype = ctypes.c_float
_libm.logf.argtypes = [ctypes.c_float]
_libm.logf.restype = ctypes.c_float


def powf(a, b):
    return F32(_libm.powf(float(F32(a)), float(F32(b))))


def test_subdomains_single_building():
    nii, njj = 9, 9
    cutk = np.zeros((nii + 2, njj + 2), F32)
    cutk[5, 5] = 2.0
    adv = OP.subdomains(cutk, nii, njj, 10.0, 20.0, 15)     # iplus = (int)(30/10) = 3, jplus = (int)(30/20) = 1
    want = np.zeros_like(adv)
    want[2:9, 4:7] = 1
    np.testing.assert_array_equal(adv, want)
    cutk[1, 9] = 2.0                                          # clipped at the domain edge
    adv = OP.subdomains(cutk, nii, njj, 10.0, 20.0, 15)
    want[1:5, 8:10] = 1
    np.testing.assert_array_equal(adv, want)


def test_subdomains_match_host_builder():
    dom = prep.small_domain(40, 36, seed=4, n_buildings=5)
    adv = OP.subdomains(dom.static.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 15)
    np.testing.assert_array_equal(adv, prep.advdom_from_cutk(dom.static.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 15))


def tiny_grid():
    nii, njj, nkk = 4, 3, 6
    dzk = np.array([0, 2, 2, 2, 4, 4, 4, 0], F32)               # DZK[0..NKK+1]
    hok = np.zeros(nkk + 2, F32)
    for k in range(1, nkk + 2):
        hok[k] = hok[k - 1] + dzk[k]
    cutk = np.zeros((nii + 2, njj + 2), F32)
    cutk[2, 2] = 4.5                                           # cell centres 1, 3, 5, ... -> levels 1, 2 inside
    grid = dict(nii=nii, njj=njj, nkk=nkk, vert_cells_ff=2, dxk=2.0, dyk=2.0, near_wall=0, igeb=1)
    return grid, cutk, dzk, hok


@pytest.mark.parametrize("ob", [1000.0, -50.0])
def test_flat_init_power_profile(ob):
    grid, cutk, dzk, hok = tiny_grid()
    nii, njj, nkk = grid["nii"], grid["njj"], grid["nkk"]
    met = MetProfile(np.array([0, 10], F32), np.array([0, 2.0], F32), np.array([0, -1.5], F32), ob)
    kk, ahk, kadv, f = OP.flat_init(grid, cutk, dzk, hok, met)
    expo = F32(0.56) * powf(ob, -0.15) if ob > 0 else max(F32(0.35) - F32(0.4) * powf(abs(ob), -0.15), F32(0.05))
    for k in range(1, nkk + 1):
        vz = hok[k - 1] + dzk[k] * F32(0.5)
        d = powf(vz / F32(10), expo)
        u, v = F32(2.0) * d, F32(-1.5) * d
        assert f.uk[1, 1, k] == u and f.vk[1, 1, k] == v
        inside = vz <= cutk[2, 2]
        assert f.uk[2, 2, k] == (0 if inside else u)
        assert f.uk[3, 2, k] == (0 if inside else u)            # face shared with the obstacle (west)
        assert f.vk[2, 3, k] == (0 if inside else v)            # (south)
        assert f.uk[nii + 1, 2, k] == f.uk[nii, 2, k]           # east edge copy
        assert f.vk[2, njj + 1, k] == f.vk[2, njj, k]           # north edge copy
        assert f.vk[nii + 1, 2, k] == 0 and f.uk[2, njj + 1, k] == 0
    assert kk[2, 2] == 2 and kk[1, 1] == 0
    assert ahk[2, 2] == hok[2] and ahk[1, 1] == 0
    assert kadv == 2 + 2
    assert not f.wk.any() and not f.uk[..., 0].any() and not f.uk[..., nkk + 1].any()


def test_flat_init_interpolation():
    grid, cutk, dzk, hok = tiny_grid()
    mh = np.array([0, 2.0, 6.0, 13.0], F32)
    ou = np.array([0, 1.0, 2.5, 4.0], F32)
    ov = np.array([0, 0.5, -0.5, 1.0], F32)
    kk, ahk, kadv, f = OP.flat_init(grid, cutk, dzk, hok, MetProfile(mh, ou, ov, 300.0))
    for k in range(1, grid["nkk"] + 1):
        vz = hok[k - 1] + dzk[k] * F32(0.5)
        if vz <= mh[1]:
            continue
        if vz > mh[3]:
            assert f.uk[1, 1, k] == ou[3] and f.vk[1, 1, k] == ov[3]
            continue
        ipo = 1 + sum(1 for q in (1, 2, 3) if vz > mh[q])
        u = ou[ipo - 1] + (ou[ipo] - ou[ipo - 1]) / (mh[ipo] - mh[ipo - 1]) * (vz - mh[ipo - 1])
        v = ov[ipo - 1] + (ov[ipo] - ov[ipo - 1]) / (mh[ipo] - mh[ipo - 1]) * (vz - mh[ipo - 1])
        assert f.uk[1, 1, k] == F32(u) and f.vk[1, 1, k] == F32(v), k


def test_flat_init_near_wall_factor():
    nii, njj, nkk = 9, 9, 6
    dzk = np.array([0, 2, 2, 2, 2, 2, 2, 0], F32)
    hok = np.cumsum(dzk).astype(F32)
    cutk = np.zeros((nii + 2, njj + 2), F32)
    cutk[3, 5] = 5.0                                           # two cells west of (5,5); centres 1, 3, 5 m inside
    grid = dict(nii=nii, njj=njj, nkk=nkk, vert_cells_ff=2, dxk=2.0, dyk=2.0, near_wall=2, igeb=3)
    met = MetProfile(np.array([0, 10], F32), np.array([0, 2.0], F32), np.array([0, 0.0], F32), 1000.0)
    kk, ahk, kadv, f = OP.flat_init(grid, cutk, dzk, hok, met)
    ref = OP.flat_init(dict(grid, near_wall=0), cutk, dzk, hok, met)[3]
    fac = F32(0.19) * F32(_libm.logf(float((F32(4.0) + F32(0.5)) * F32(10))))   # obstacle 2 cells = 4 m away
    for k in range(1, nkk):
        vz = hok[k - 1] + dzk[k] * F32(0.5)
        want = ref.uk[5, 5, k] * fac if vz <= ahk[3, 5] else ref.uk[5, 5, k]
        assert f.uk[5, 5, k] == want, k
    assert kk[3, 5] == 3 and ahk[3, 5] == hok[3]


def test_vegetation_rule_and_order():
    nii, njj, nkk = 4, 4, 8
    dzk = np.array([0] + [2] * nkk + [0], F32)
    hok = np.cumsum(dzk).astype(F32)
    kkart = np.zeros((nii + 2, njj + 2), np.int16)
    kkart[2, 2] = 1
    pts = [dict(crown_height=10.0, trunk_height=3.0, trunk_lad=0.2, crown_lad=0.8, cov=0.5, i=2, j=2, drag=1),
           dict(crown_height=5.0, trunk_height=1.0, trunk_lad=0.1, crown_lad=0.4, cov=0.9, i=2, j=2, drag=1),
           dict(crown_height=8.0, trunk_height=2.0, trunk_lad=0.3, crown_lad=0.6, cov=0.7, i=3, j=1, drag=0),
           dict(crown_height=8.0, trunk_height=2.0, trunk_lad=0.3, crown_lad=0.6, cov=0.7, i=9, j=1, drag=1)]
    cov0 = np.full((nii + 2, njj + 2), 0.25, F32)
    veg, mask, cov = OP.vegetation(nii, njj, nkk, kkart, dzk, hok, pts, cov0)
    for k in range(nkk):
        mch = hok[k] - hok[1] + dzk[k] * F32(0.5)
        want = F32(0)
        for p in pts[:2]:
            if float(mch) < p["crown_height"]:
                lad = p["trunk_lad"] if (mch >= 0 and float(mch) < p["trunk_height"]) else p["crown_lad"]
                if mch >= 0:
                    want = F32(0.3 * math.pow(p["cov"], 3) * lad)
        assert veg[2, 2, k] == want, k
    assert mask[2, 2] == 1 and mask[3, 1] == 0 and mask.sum() == 1
    assert cov[2, 2] == F32(0.9) and cov[3, 1] == F32(0.7) and cov[1, 1] == F32(0.25)
    assert not veg[3, 1].any()
