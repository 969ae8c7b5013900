"""GPU parity of the flow-field set-up: device entry points against ``oracle/prep.cpp``.

``gral_prog_subdomains``, ``gral_prog_flat_init`` and ``gral_prog_vegetation`` must give exactly
the oracle's arrays (ADVDOM; KKART, AHK, KADVMAX and the initial U/V/W; VEG, its mask and COV)
on: small and production-size (400x400x63) grids, one and three measurement heights, stable and
unstable profiles, per-column Obukhov lengths, both near-wall damping modes, and vegetation with
several lines per cell, lines outside the grid and lines that set COV only.  Bit-identical
integer and float results are the bar.
"""
import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.abi import MetProfile
from gral_b200.prognostic import PrognosticSolver
from oracle import prep as OP

pytestmark = pytest.mark.gpu

F32 = np.float32


def same(a, b):
    np.testing.assert_array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def grid_of(dom, near_wall=0, igeb=None):
    ig = max(int(20 / dom.dxk), 1) if igeb is None else igeb
    return dict(nii=dom.nii, njj=dom.njj, nkk=dom.nkk, vert_cells_ff=dom.vert_cells_ff, dxk=dom.dxk, dyk=dom.dyk,
                near_wall=near_wall, igeb=ig)


METS = {
    "stable_1h": MetProfile(np.array([0, 10], F32), np.array([0, 2.3], F32), np.array([0, -1.1], F32), 250.0),
    "unstable_1h": MetProfile(np.array([0, 10], F32), np.array([0, -3.0], F32), np.array([0, 0.7], F32), -40.0),
    "three_heights": MetProfile(np.array([0, 3.0, 12.0, 40.0], F32), np.array([0, 1.0, 2.2, 3.5], F32),
                                np.array([0, -0.4, -1.0, -2.5], F32), 1000.0),
}


def check_flat(s, dom, grid, met, advdom=None):
    st = dom.static
    got = s.flat_init(grid, st.cutk, st.dzk, st.hokart, met, advdom)
    want = OP.flat_init(grid, st.cutk, st.dzk, st.hokart, met, advdom)
    same(got[0], want[0])
    same(got[1], want[1])
    assert got[2] == want[2]
    for name in ("uk", "vk", "wk"):
        same(getattr(got[3], name), getattr(want[3], name))
    return got


@pytest.mark.parametrize("met", list(METS))
def test_flat_init_small(gpu_required, met):
    dom = prep.small_domain(40, 36, seed=9, n_buildings=6)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        kk, ahk, kadv, f = check_flat(s, dom, grid_of(dom), METS[met])
        # the set-up's KKART and KADVMAX are the ones the domain builder uses for the solve
        same(kk, dom.static.kkart)
        assert kadv == dom.kadvmax


def test_flat_init_adaptive_and_near_wall(gpu_required):
    dom = prep.small_domain(48, 44, seed=12, n_buildings=7)
    rng = np.random.default_rng(5)
    ol = rng.choice(np.array([-80.0, -15.0, 60.0, 400.0, 1000.0], F32), size=(dom.nii + 2, dom.njj + 2)).astype(F32)
    met = MetProfile(METS["stable_1h"].heights, METS["stable_1h"].obs_u, METS["stable_1h"].obs_v, 250.0, ol)
    adv = OP.subdomains(dom.static.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 2)   # small sub-domains
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        check_flat(s, dom, grid_of(dom), met)
        for mode in (1, 2):
            check_flat(s, dom, grid_of(dom, near_wall=mode, igeb=4), METS["unstable_1h"], adv)


def test_subdomains(gpu_required):
    for seed, factor in ((1, 15), (2, 3), (3, 0)):
        dom = prep.small_domain(60, 52, seed=seed, n_buildings=5)
        with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
            got = s.subdomains(dom.static.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, factor)
        same(got, OP.subdomains(dom.static.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, factor))


def veg_lines(dom, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        crown = float(rng.uniform(2.0, 25.0))
        out.append(dict(crown_height=crown, trunk_height=crown * float(rng.uniform(0, 60)) * 0.01,
                        trunk_lad=float(rng.uniform(0.05, 0.5)), crown_lad=float(rng.uniform(0.1, 1.5)),
                        cov=float(rng.uniform(0.1, 1.0)), i=int(rng.integers(-2, dom.nii + 4)),
                        j=int(rng.integers(-2, dom.njj + 4)), drag=int(rng.random() < 0.85)))
    # several lines on the same cells, in file order
    for q in range(0, n // 4):
        out.append(dict(out[q], crown_height=out[q]["crown_height"] * 0.5, cov=0.33))
    return out


def test_vegetation(gpu_required):
    dom = prep.small_domain(40, 36, seed=3, n_buildings=5)
    st = dom.static
    pts = veg_lines(dom, 600, seed=8)
    cov0 = np.full((dom.nii + 2, dom.njj + 2), 0.1, F32)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        got = s.vegetation(dom.nii, dom.njj, dom.nkk, st.kkart, st.dzk, st.hokart, pts, cov0)
        want = OP.vegetation(dom.nii, dom.njj, dom.nkk, st.kkart, st.dzk, st.hokart, pts, cov0)
        for a, b in zip(got, want):
            same(a, b)
        assert got[1].sum() > 100
        # no lines: VEG all zero, COV unchanged
        got = s.vegetation(dom.nii, dom.njj, dom.nkk, st.kkart, st.dzk, st.hokart, [], cov0)
        assert not got[0].any() and not got[1].any()
        same(got[2], cov0)


def test_production_grid(gpu_required):
    """400x400x63 city grid: sub-domains, set-up with near-wall damping, vegetation."""
    dom = prep.city_domain()
    st = dom.static
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        adv = s.subdomains(st.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 15)
        same(adv, st.advdom)
        kk, ahk, kadv, f = check_flat(s, dom, grid_of(dom, near_wall=1), METS["three_heights"], adv)
        same(kk, st.kkart)
        pts = veg_lines(dom, 20000, seed=2)
        cov0 = np.zeros((dom.nii + 2, dom.njj + 2), F32)
        got = s.vegetation(dom.nii, dom.njj, dom.nkk, kk, st.dzk, st.hokart, pts, cov0)
        want = OP.vegetation(dom.nii, dom.njj, dom.nkk, kk, st.dzk, st.hokart, pts, cov0)
        for a, b in zip(got, want):
            same(a, b)


def test_rejects(gpu_required):
    dom = prep.small_domain(16, 14, seed=1)
    st = dom.static
    from gral_b200.prognostic import GralError
    from gral_b200 import abi
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for bad in (dict(grid_of(dom), nii=dom.nii + 1), dict(grid_of(dom), near_wall=3),
                    dict(grid_of(dom), near_wall=1)):       # near_wall 1 without ADVDOM
            with pytest.raises(GralError) as e:
                s.flat_init(bad, st.cutk, st.dzk, st.hokart, METS["stable_1h"])
            assert e.value.code == abi.GRAL_EINVAL
        empty = MetProfile(np.zeros(1, F32), np.zeros(1, F32), np.zeros(1, F32), 100.0)
        with pytest.raises(GralError):
            s.flat_init(grid_of(dom), st.cutk, st.dzk, st.hokart, empty)
        # still usable
        check_flat(s, dom, grid_of(dom), METS["stable_1h"])
