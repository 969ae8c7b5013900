"""Edge cases of the solver against the oracle: the deepest slab the column kernels take (KADVMAX
62, i.e. 64 levels in two rounds of 32 lanes), the smallest grids whose sweep rectangles are only a
few columns wide, and a KADVMAX beyond the slab, which must be rejected before any GPU work.
Both layouts (slab and interleaved) and turbulence models 1 and 2; bit-identical fields."""
import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.prognostic import GralError, PrognosticSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["slab", "interleaved"])
def layout(request, monkeypatch):
    monkeypatch.setenv("GRAL_PROG_LAYOUT", request.param)
    return request.param


def deepest_domain():
    km = int(prep.small_domain(14, 12, seed=3, n_buildings=2, vert_cells_ff=12).static.kkart.max())
    d = prep.small_domain(14, 12, seed=3, n_buildings=2, vert_cells_ff=62 - km)
    assert d.kadvmax == 62
    return d


def tiny_domain():
    return prep.make_domain(6, 5, 2.0, 2.0, 1.05, 8, [prep.Building(2, 3, 2, 2, 6.0)])


def check(dom, model, layout):
    sits = [prep.Situation(direction_deg=230.0), prep.Situation(direction_deg=40.0, speed_10m=4.0)]
    ps = [dom.params(x, model=model, iterations=4) for x in sits]
    f0 = [prep.initial_fields(dom, x, model) for x in sits]
    fg = [f.copy() for f in f0]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(sits)) as s:
        st = s.calculate_batch(ps, dom.static, fg)
    assert st[0]["layout"] == (1 if layout == "interleaved" else 0)
    for b in range(len(sits)):
        fc = f0[b].copy()
        O.solve(ps[b], dom.static, fc)
        for name in ("uk", "vk", "wk"):
            np.testing.assert_array_equal(getattr(fg[b], name), getattr(fc, name), err_msg=(b, name))


@pytest.mark.parametrize("model", [1, 2])
def test_deepest_slab(gpu_required, layout, model):
    check(deepest_domain(), model, layout)


@pytest.mark.parametrize("model", [1, 2])
def test_tiny_grid(gpu_required, layout, model):
    check(tiny_domain(), model, layout)


def test_slab_too_deep_is_rejected(gpu_required):
    d = deepest_domain()
    p = d.params(prep.Situation(), iterations=2)
    p["kadvmax"] = 63
    f = prep.initial_fields(d, prep.Situation())
    with PrognosticSolver(d.nii, d.njj, d.nkk, 63) as s:
        with pytest.raises(GralError) as e:
            s.calculate(p, d.static, f)
    assert e.value.code == abi.GRAL_EINVAL
