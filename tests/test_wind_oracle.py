"""The CPU restatement of Zeitschleife.IntWindCalculate (``oracle/wind.cpp``) on known answers.

Fields built so the expected result is known in closed form: a field linear in i (and j) gives
the face interpolation exactly, the level index is the first HOKART at or above the height in
both the binary (terrain) and the linear (flat, buildings) search, W is interpolated with the
level's DZK, and the profile branch uses the C library's powf below/above one height and the
linear rule between three.
"""
import ctypes
import ctypes.util

import numpy as np
import pytest

from gral_b200.abi import PARTICLE_DTYPE, FieldArrays, MetProfile
from oracle import prep as OP

F32 = np.float32
_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.powf.restype = ctypes.c_float


def grid_fields(nii=6, njj=5, nkk=12):
    dzk = np.array([0] + [2.0 + 0.5 * k for k in range(1, nkk + 1)] + [0], F32)
    hok = np.zeros(nkk + 2, F32)
    for k in range(1, nkk + 2):
        hok[k] = hok[k - 1] + dzk[k]
    shape = (nii + 2, njj + 2, nkk + 2)
    i, j, k = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), np.arange(shape[2]), indexing="ij")
    f = FieldArrays((1.5 * i + 0.01 * k).astype(F32), (-0.5 * j + 0.02 * k).astype(F32), (0.1 * k).astype(F32))
    return nii, njj, nkk, dzk, hok, f


def particles(rows):
    return np.array(rows, dtype=PARTICLE_DTYPE)


@pytest.mark.parametrize("terrain", [0, 1])
def test_level_index_and_faces(terrain):
    nii, njj, nkk, dzk, hok, f = grid_fields()
    g = dict(terrain=terrain, buildings=1, ikooa=100, jkooa=-40, dxk=2.0, dyk=4.0, ahmin=0.0)
    zs = [0.5, hok[3], hok[3] + 0.01, hok[nkk] - 0.1, hok[nkk] + 50.0]
    p = particles([(100 + 2 * 2 + 0.5, -40 + 4 * 1 + 1.0, z, 0.0, 3, 2) for z in zs])
    ux, uy, uz, kk = OP.wind_at(g, nii, njj, nkk, dzk, hok, f, p)
    for q, z in enumerate(zs):
        k = next((k for k in range(1, nkk + 1) if hok[k] >= F32(z)), nkk)
        assert kk[q] == k
        u1, u2 = f.uk[3, 2, k], f.uk[4, 2, k]
        base = F32(100) + F32(2) * F32(2.0)
        want = F32(float(u1) + float((u2 - u1) / F32(2.0)) * (p["x"][q] - float(base)))
        assert ux[q] == want
        w1, w2 = f.wk[3, 2, k], f.wk[3, 2, k + 1]
        assert uz[q] == w1 + (w2 - w1) / dzk[k] * (F32(z) + F32(0) - hok[k - 1])


def test_profile_branch():
    met1 = MetProfile(np.array([0, 10.0], F32), np.array([0, 3.0], F32), np.array([0, -1.0], F32), 300.0)
    g = dict(terrain=0, buildings=0, dxk=2.0, dyk=2.0, met=None)
    zs = [2.0, 10.0, 35.0]
    p = particles([(0.0, 0.0, z, 0.0, 1, 1) for z in zs])
    ux, uy, uz, kk = OP.wind_at(g, 4, 4, 4, None, None, None, p, met1)
    e = F32(0.56) * F32(_libm.powf(300.0, -0.15))
    for q, z in enumerate(zs):
        d = F32(_libm.powf(float(F32(z) / F32(10.0)), float(e)))
        assert ux[q] == F32(3.0) * d and uy[q] == F32(-1.0) * d and uz[q] == 0 and kk[q] == 0
    met3 = MetProfile(np.array([0, 2.0, 8.0, 20.0], F32), np.array([0, 1.0, 2.0, 4.0], F32),
                      np.array([0, 0.5, 0.25, -1.0], F32), -30.0)
    p = particles([(0.0, 0.0, 5.0, 0.0, 1, 1), (0.0, 0.0, 20.0, 0.0, 1, 1)])
    ux, uy, uz, kk = OP.wind_at(g, 4, 4, 4, None, None, None, p, met3)
    help_ = F32(1) / (F32(8.0) - F32(2.0)) * (F32(5.0) - F32(2.0))
    assert ux[0] == F32(1.0) + (F32(2.0) - F32(1.0)) * help_
    assert ux[1] == F32(4.0) and uy[1] == F32(-1.0)          # at or above the top height: its value
