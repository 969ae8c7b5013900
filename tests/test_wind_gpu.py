"""GPU parity of the wind at particle positions (``gral_prog_wind_at``) against ``oracle/wind.cpp``.

After a solve, particles spread over the grid and the column (including heights below the first
level, at level tops and above the top) are interpolated on the device from the resident fields
and by the CPU restatement from the fields ``gral_prog_store`` returned: the terrain (binary
search) and flat-with-buildings branches must agree bit for bit, U, V, W and IndexK; the met
profile branch within two units in the last place (the device evaluates the power law with a
double-precision pow rounded to float, within one unit of the reference's C-library powf, and
multiplies it by the wind component).
"""
import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.abi import PARTICLE_DTYPE, MetProfile
from gral_b200.prognostic import GralError, PrognosticSolver
from oracle import prep as OP

pytestmark = pytest.mark.gpu

F32 = np.float32


def random_particles(dom, n, seed, ikooa, jkooa):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["i"] = rng.integers(1, dom.nii + 1, n)
    p["j"] = rng.integers(1, dom.njj + 1, n)
    p["x"] = ikooa + (p["i"] - 1) * dom.dxk + rng.uniform(0, dom.dxk, n)
    p["y"] = jkooa + (p["j"] - 1) * dom.dyk + rng.uniform(0, dom.dyk, n)
    top = float(dom.static.hokart[dom.nkk])
    z = rng.uniform(-1.0, top * 1.1, n).astype(F32)
    z[: n // 10] = dom.static.hokart[rng.integers(0, dom.nkk + 1, n // 10)]      # exactly at level tops
    p["z"] = z
    p["ahint"] = rng.uniform(0, 3.0, n).astype(F32)
    return p


def solved(dom, sit):
    f = prep.initial_fields(dom, sit)
    s = PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax)
    s.load([dom.params(sit, iterations=4)], dom.static, [f])
    s.iterate()
    s.store([f])
    return s, f


def ulp_diff(a, b):
    """Units in the last place between equal-signed floats; NaN must sit in the same places (a
    particle below ground gives a negative base of the power law, NaN on both sides)."""
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    ai = a[~na].view(np.int32).astype(np.int64)
    bi = b[~nb].view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


@pytest.mark.parametrize("terrain", [0, 1])
def test_field_branches(gpu_required, terrain):
    dom = prep.small_domain(24, 20, seed=6, n_buildings=4)
    s, f = solved(dom, prep.Situation(direction_deg=240.0))
    with s:
        g = dict(terrain=terrain, buildings=1, ikooa=312000, jkooa=5160000, dxk=dom.dxk, dyk=dom.dyk,
                 ahmin=0.75 if terrain else 0.0)
        p = random_particles(dom, 20000, seed=terrain, ikooa=g["ikooa"], jkooa=g["jkooa"])
        got = s.wind_at(0, g, dom.static.dzk, dom.static.hokart, p)
        want = OP.wind_at(g, dom.nii, dom.njj, dom.nkk, dom.static.dzk, dom.static.hokart, f, p)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        assert len(np.unique(got[3])) > dom.nkk // 2


def test_profile_branch(gpu_required):
    dom = prep.small_domain(16, 14, seed=1)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for met in (MetProfile(np.array([0, 10.0], F32), np.array([0, 2.5], F32), np.array([0, -1.2], F32), -60.0),
                    MetProfile(np.array([0, 3.0, 15.0, 50.0], F32), np.array([0, 1.0, 2.0, 4.0], F32),
                               np.array([0, 0.3, -0.2, -1.0], F32), 400.0)):
            g = dict(terrain=0, buildings=0, dxk=dom.dxk, dyk=dom.dyk)
            p = random_particles(dom, 50000, seed=3, ikooa=0, jkooa=0)
            got = s.wind_at(0, g, None, None, p, met)
            want = OP.wind_at(g, dom.nii, dom.njj, dom.nkk, None, None, None, p, met)
            # the power-law factor within 1 ulp of powf; after the product with the wind
            # component U and V within 2 ulp
            assert ulp_diff(got[0], want[0]).max() <= 2 and ulp_diff(got[1], want[1]).max() <= 2
            ok = ~np.isnan(want[0])
            assert ok.mean() > 0.9
            exact = float((got[0][ok] == want[0][ok]).mean())
            assert exact > 0.99, exact
            assert not got[2].any() and not got[3].any()


def test_rejects_and_production(gpu_required):
    dom = prep.city_domain()
    sit = prep.Situation(direction_deg=225.0, speed_10m=2.0, z0=0.5)
    s, f = solved(dom, sit)
    with s:
        g = dict(terrain=0, buildings=1, ikooa=0, jkooa=0, dxk=dom.dxk, dyk=dom.dyk)
        p = random_particles(dom, 1 << 20, seed=9, ikooa=0, jkooa=0)
        got = s.wind_at(0, g, dom.static.dzk, dom.static.hokart, p)
        want = OP.wind_at(g, dom.nii, dom.njj, dom.nkk, dom.static.dzk, dom.static.hokart, f, p)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        bad = p[:8].copy()
        bad["i"][3] = dom.nii + 1
        with pytest.raises(GralError) as e:
            s.wind_at(0, g, dom.static.dzk, dom.static.hokart, bad)
        assert e.value.code == abi.GRAL_EINVAL
        with pytest.raises(GralError) as e:
            s.wind_at(1, g, dom.static.dzk, dom.static.hokart, p[:8])
        assert e.value.code == abi.GRAL_EINVAL
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s2:
        with pytest.raises(GralError) as e:
            s2.wind_at(0, g, dom.static.dzk, dom.static.hokart, p[:8])
        assert e.value.code == abi.GRAL_ESTATE
