"""Input builders (gral_b200.prep) against the grid rules of the reference and the named
workload shapes: vertical grid (ProgramFunctions.cs:27-77), KKART/KADVMAX (MicroscaleFlat.cs:56-197),
ADVDOM sub-domains (ReadGeometryAndDomains.cs:321-347) and VerticalIndex
(PrognosticFlowfield.cs:339)."""
import numpy as np
import pytest

from gral_b200 import prep


def vertical_index(dom):
    kk = dom.static.kkart.astype(np.int32)
    return np.minimum(dom.nkk - 1, kk + dom.vert_cells_ff)


def test_cube_domain_100x100():
    """100x100 cells at 2 m, first layer 2 m, stretch 1.01: NKK 162 with the top near 802.5 m;
    the 20 m cube gives KKART 10 and KADVMAX 30; VerticalIndex 20 in the open, 30 at the cube."""
    d = prep.cube_domain()
    assert (d.nii, d.njj, d.nkk, d.kadvmax) == (100, 100, 162, 30)
    assert abs(float(d.static.hokart[d.nkk]) - 802.5) < 0.1
    assert int(d.static.kkart.max()) == 10
    cube = d.static.cutk > 0
    assert cube.sum() == 100 and np.array_equal(np.argwhere(cube).min(0), [46, 46])
    vi = vertical_index(d)[1:-1, 1:-1]
    assert set(np.unique(vi)) == {20, 30}
    assert d.static.advdom[1:-1, 1:-1].min() == 1


def test_city_domain_400x400():
    """400x400 at 2 m, stretch 1.05: NKK 63; 64 buildings 10-30 m tall with 10-40 m footprints;
    KKART 5/8/11 for 10/20/30 m heights; VerticalIndex at most 41 = KADVMAX."""
    d = prep.city_domain()
    assert (d.nii, d.njj, d.nkk) == (400, 400, 63)
    assert len(d.buildings) == 64
    for b in d.buildings:
        assert 10.0 <= b.height <= 30.0
        assert 10 <= (b.i1 - b.i0 + 1) * 2 <= 40 and 10 <= (b.j1 - b.j0 + 1) * 2 <= 40
    kk = prep.kkart_from_cutk(np.array([[10.0, 20.0, 30.0]], np.float32), d.static.dzk, d.static.hokart, d.nkk)
    assert kk.tolist() == [[5, 8, 11]]
    assert vertical_index(d)[1:-1, 1:-1].max() == d.kadvmax == 41


def test_buildings_do_not_overlap():
    d = prep.city_domain()
    occ = np.zeros((d.nii + 2, d.njj + 2), np.int32)
    for b in d.buildings:
        occ[b.i0:b.i1 + 1, b.j0:b.j1 + 1] += 1
    assert occ.max() == 1


def test_builders_are_seeded():
    a, b = prep.city_domain(), prep.city_domain()
    assert np.array_equal(a.static.cutk, b.static.cutk)
    c = prep.small_domain(16, 14, seed=0)
    e = prep.small_domain(16, 14, seed=1)
    assert not np.array_equal(c.static.cutk, e.static.cutk)


@pytest.mark.parametrize("direction", [0.0, 90.0, 225.0, 270.0])
def test_initial_fields_log_profile(direction):
    """10 m speed equals the requested speed in the free stream; zero inside obstacles and on
    faces shared with an obstacle; U/V follow the meteorological direction."""
    d = prep.small_domain(16, 14, seed=0)
    sit = prep.Situation(direction_deg=direction, speed_10m=3.0, z0=0.2)
    f = prep.initial_fields(d, sit)
    st = d.static
    z = st.hokart[0:d.nkk] + st.dzk[1:d.nkk + 1] * np.float32(0.5)
    open_ij = np.argwhere(st.cutk[1:-1, 1:-1] == 0)[0] + 1
    i, j = open_ij
    speed = np.hypot(f.uk[i, j, 1:d.nkk + 1], f.vk[i, j, 1:d.nkk + 1]).astype(np.float64)
    s10 = np.interp(10.0, z.astype(np.float64), speed)
    assert abs(s10 - 3.0) < 0.05
    th = np.radians(direction)
    k = d.nkk // 2
    assert np.sign(np.round(f.uk[i, j, k], 4)) == np.sign(np.round(-np.sin(th), 4))
    inside = z[None, None, :] <= st.cutk[:, :, None]
    assert not f.uk[:, :, 1:d.nkk + 1][inside].any()
    assert not f.vk[:, :, 1:d.nkk + 1][inside].any()
    assert f.turb is None and prep.initial_fields(d, sit, 2).turb is not None


def test_params_reference_scalars():
    d = prep.small_domain(16, 14, seed=0)
    p = d.params(prep.Situation(ustar=0.25), model=2, iterations=7)
    assert p["turbulence_model"] == 2 and p["iteration_steps_max"] == 7
    assert p["v0_1"] == np.float32(0.5)
    # CorolisParam of the reference for 47 deg latitude, float32
    assert abs(p["coriolis"] - 2 * 7.29e-5 * np.sin(47 * 3.1415 / 180)) < 1e-9


def test_hilly_domains_build():
    """The uneven-domain instances build for small and large grids: hills raise KKART, every
    column of a hilly grid is prognostic, KADVMAX follows KKART + VertCellsFF."""
    for q, (ni, nj, dx, vc) in enumerate([(20, 20, 2.0, 8), (24, 20, 2.0, 8), (48, 28, 4.0, 9), (128, 112, 2.0, 20),
                                          (192, 176, 2.5, 30)]):
        d = prep.hilly_domain(ni, nj, dx, vc, seed=q)
        st = d.static
        assert d.kadvmax == min(d.nkk, max(1, int(st.kkart[st.cutk > 0].max())) + vc)
        assert st.kkart.max() > 0
        assert (st.cutk[1:ni + 1, 1:nj + 1] > 0).all()
