"""The load that builds the initial fields on the device (``gral_prog_load_flat``).

Loading the flat-terrain set-up's fields from the host (computed by the oracle's restatement of
MicroscaleFlat.cs) and building them on the device from the same met profiles must give the same
solve bit for bit: slab and interleaved layouts, one and three measurement heights, with and
without the near-wall damping, model 1 and model 2; and the same as the oracle's solve.
"""
import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.abi import FieldArrays, MetProfile
from gral_b200.prognostic import GralError, PrognosticSolver
from oracle import oracle as O
from oracle import prep as OP

pytestmark = pytest.mark.gpu

F32 = np.float32


def met_of(q):
    if q % 2 == 0:
        return MetProfile(np.array([0, 10.0], F32), np.array([0, 1.5 + 0.3 * q], F32),
                          np.array([0, -1.0 + 0.2 * q], F32), [250.0, -40.0, 800.0][q % 3])
    return MetProfile(np.array([0, 3.0, 12.0, 40.0], F32), np.array([0, 1.0, 2.0 + 0.1 * q, 3.5], F32),
                      np.array([0, 0.4, -0.3, -1.0 - 0.1 * q], F32), 1000.0)


def grid_of(dom, near_wall):
    return dict(nii=dom.nii, njj=dom.njj, nkk=dom.nkk, vert_cells_ff=dom.vert_cells_ff, dxk=dom.dxk, dyk=dom.dyk,
                near_wall=near_wall, igeb=4)


def empty_fields(dom, model):
    shape = (dom.nii + 2, dom.njj + 2, dom.nkk + 2)
    z = lambda: np.zeros(shape, F32)
    return FieldArrays(z(), z(), z(), z() if model != 1 else None, z() if model != 1 else None)


@pytest.mark.parametrize("n,near_wall,model", [(2, 0, 1), (3, 1, 1), (33, 0, 1), (2, 2, 2)])
def test_load_flat_matches_host_fields(gpu_required, n, near_wall, model):
    dom = prep.small_domain(40, 36, seed=9, n_buildings=6)
    st = dom.static
    grid = grid_of(dom, near_wall)
    mets = [met_of(q) for q in range(n)]
    host = []
    for m in mets:
        kk, ahk, kadv, f = OP.flat_init(grid, st.cutk, st.dzk, st.hokart, m, st.advdom)
        np.testing.assert_array_equal(kk, st.kkart)
        assert kadv == dom.kadvmax
        if model != 1:
            f.turb = np.zeros_like(f.uk)
            f.tdiss = np.zeros_like(f.uk)
        host.append(f)
    ps = [dom.params(None, model=model, iterations=8) for _ in range(n)]
    a = [f.copy() for f in host]
    b = [empty_fields(dom, model) for _ in range(n)]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=n) as s:
        s.load(ps, st, a)
        s.iterate()
        sa = s.store(a)
        s.load_flat(ps, st, mets, grid, b)
        s.iterate()
        sb = s.store(b)
    for q in range(n):
        for name in ("uk", "vk", "wk"):
            np.testing.assert_array_equal(getattr(a[q], name), getattr(b[q], name), err_msg=(q, name))
        assert sa[q]["iterations"] == sb[q]["iterations"] and sa[q]["dtime"] == sb[q]["dtime"]
        assert sa[q]["topwind"] == sb[q]["topwind"]
    if n <= 3:   # and the oracle's solve of the host fields
        want = host[0].copy()
        O.solve(ps[0], st, want)
        np.testing.assert_array_equal(b[0].uk, want.uk)


def test_load_flat_rejects(gpu_required):
    dom = prep.small_domain(24, 20, seed=2)
    st = dom.static
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for bad in (dict(grid_of(dom, 0), nii=dom.nii - 1), dict(grid_of(dom, 0), dxk=dom.dxk * 2),
                    dict(grid_of(dom, 0), near_wall=5)):
            with pytest.raises(GralError) as e:
                s.load_flat([dom.params(None, iterations=2)], st, [met_of(0)], bad, [empty_fields(dom, 1)])
            assert e.value.code == abi.GRAL_EINVAL
