"""GPU parity: the CUDA solver (through the C ABI) against the CPU oracle on the same inputs.

Both implement the reference's deterministic float32 evaluation order, so the expected difference
is zero; asserted are the north-star bound max|dU|/max|U| <= 1e-4 on U, V, W, bit-identical
fields, identical DeltaUMax traces and identical iteration counts and convergence decisions.
Both kernel families are covered: the slab layout (one warp per column, few situations) and the
interleaved layout (lane per situation, batches), forced with GRAL_PROG_LAYOUT.
"""
import os

import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.prognostic import PrognosticSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


def rel_err(a, b):
    den = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max()) / den


@pytest.fixture(params=["slab", "interleaved"])
def layout(request, monkeypatch):
    monkeypatch.setenv("GRAL_PROG_LAYOUT", request.param)
    return request.param


def solve_gpu(dom, params, fields, traces=None):
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(params)) as s:
        return s.calculate_batch(params, dom.static, fields, traces)


def check_same(fg, fc, names=("uk", "vk", "wk")):
    for name in names:
        a, b = getattr(fg, name), getattr(fc, name)
        assert rel_err(a, b) <= TOL, name
        assert np.array_equal(a, b), f"{name} not bit-identical (max rel err {rel_err(a, b):.3e})"


def run_pair(dom, sits, iterations, model=1, **kw):
    ps = [dom.params(x, model=model, iterations=iterations, **kw) for x in sits]
    f0 = [prep.initial_fields(dom, x, model) for x in sits]
    fg = [f.copy() for f in f0]
    tg = [np.zeros(max(iterations, 1), np.float32) for _ in sits]
    sg = solve_gpu(dom, ps, fg, tg)
    out = []
    for b, x in enumerate(sits):
        fc = f0[b].copy()
        tc = np.zeros(max(iterations, 1), np.float32)
        sc = O.solve(ps[b], dom.static, fc, tc)
        out.append((fg[b], fc, sg[b], sc, tg[b], tc))
    return out


@pytest.mark.parametrize("iterations", [1, 2, 4, 9])
@pytest.mark.parametrize("seed", [0, 1])
def test_model1_small(gpu_required, layout, seed, iterations):
    dom = prep.small_domain(16, 14, seed=seed)
    sit = prep.Situation(direction_deg=250.0 + 30 * seed, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], iterations):
        assert sg["iterations"] == sc["iterations"] == iterations
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


def test_model1_batch_mixed_directions(gpu_required, layout):
    """Three situations in one batch, each against its own oracle run (sweep direction, inflow
    side and boundary events differ per situation)."""
    dom = prep.small_domain(18, 15, seed=2, n_buildings=4)
    sits = [prep.Situation(direction_deg=d, speed_10m=v, z0=0.3, ustar=0.25)
            for d, v in ((15.0, 2.0), (135.0, 4.0), (290.0, 1.0))]
    for fg, fc, sg, sc, tg, tc in run_pair(dom, sits, 7):
        assert sg["iterations"] == sc["iterations"] == 7
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


def test_model1_vegetation(gpu_required, layout):
    dom = prep.small_domain(16, 16, seed=3, with_veg=True)
    assert dom.static.veg_mask.sum() > 0
    sit = prep.Situation(direction_deg=200.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], 6):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


def test_model1_convergence_decisions(gpu_required, layout):
    """The cadence test (every 100 iterations, threshold on DeltaMean/topwind^2) stops both solvers
    at the same iteration with the same residual history."""
    dom = prep.small_domain(14, 12, seed=4, n_buildings=2)
    sit = prep.Situation(direction_deg=260.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    [(fg, fc, sg, sc, tg, tc)] = run_pair(dom, [sit], 400, iter_min=100, conv_threshold=0.05)
    assert sg["iterations"] == sc["iterations"]
    assert sg["iteration_loops"] == sc["iteration_loops"]
    assert sg["converged"] == sc["converged"]
    assert sg["delta_history"] == sc["delta_history"]
    assert sg["delta_first"] == sc["delta_first"] and sg["delta_finish"] == sc["delta_finish"]
    assert sg["convergence_problem"] == sc["convergence_problem"]
    assert (sg["uk_unrealistic"], sg["vk_unrealistic"], sg["wk_unrealistic"]) == \
        (sc["uk_unrealistic"], sc["vk_unrealistic"], sc["wk_unrealistic"])
    assert sg["geschw_max"] == sc["geschw_max"]
    check_same(fg, fc)


def test_cube_domain_config1_geometry(gpu_required, layout):
    """The 100x100 cube case (2 m cells, 20 m building, stretch 1.01: NKK 162, KADVMAX 30)."""
    dom = prep.cube_domain()
    assert (dom.nkk, dom.kadvmax, int(dom.static.kkart.max())) == (162, 30, 10)
    sit = prep.Situation(direction_deg=270.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], 5):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


def test_quantise_off(gpu_required, layout):
    """quantise=0 switches the Frund rounding off on both sides."""
    dom = prep.small_domain(16, 14, seed=5)
    sit = prep.Situation(direction_deg=45.0, speed_10m=2.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], 5, quantise=0):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


@pytest.mark.parametrize("iterations", [1, 3, 8])
def test_model2_ke_small(gpu_required, layout, iterations):
    """k-epsilon closure (TurbulenceModel 2): momentum with TURB-based viscosity, the TKE/TDISS
    sweep with its wall functions and clamps, and the TURB initialisation."""
    dom = prep.small_domain(16, 14, seed=6, obukhov=-80.0)      # unstable: the BdLayHeight branch
    sit = prep.Situation(direction_deg=230.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], iterations, model=2):
        assert sg["iterations"] == sc["iterations"] == iterations
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc, ("uk", "vk", "wk", "turb", "tdiss"))


def test_model2_batch_mixed(gpu_required, layout):
    dom = prep.small_domain(18, 15, seed=7, n_buildings=4, obukhov=200.0)
    sits = [prep.Situation(direction_deg=d, speed_10m=v, z0=0.3, ustar=0.25)
            for d, v in ((20.0, 2.0), (140.0, 4.0), (300.0, 1.5))]
    for fg, fc, sg, sc, tg, tc in run_pair(dom, sits, 5, model=2):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc, ("uk", "vk", "wk", "turb", "tdiss"))


def test_model2_vegetation(gpu_required, layout):
    dom = prep.small_domain(16, 16, seed=8, with_veg=True)
    sit = prep.Situation(direction_deg=110.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], 5, model=2):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc, ("uk", "vk", "wk", "turb", "tdiss"))


@pytest.mark.parametrize("iterations", [1, 4])
def test_model0_mixing_length(gpu_required, layout, iterations):
    """TurbulenceModel 0: scalar mixing-length momentum with the double-precision W solve."""
    dom = prep.small_domain(16, 14, seed=9)
    sit = prep.Situation(direction_deg=320.0, speed_10m=2.5, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], iterations, model=0):
        assert sg["iterations"] == sc["iterations"] == iterations
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


@pytest.mark.parametrize("with_veg", [False, True])
def test_model1_vector512_width(gpu_required, layout, with_veg):
    """simd_width 16: the reference's Vector512 routines (chunks of 16 levels, fused multiply-adds
    in the power law, the height above KKART and the neighbour sums)."""
    dom = prep.small_domain(16, 16, seed=14, vert_cells_ff=20, with_veg=with_veg)
    sits = [prep.Situation(direction_deg=d, speed_10m=3.0, z0=0.2, ustar=0.3) for d in (75.0, 300.0)]
    for fg, fc, sg, sc, tg, tc in run_pair(dom, sits, 6, simd_width=16):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc)


def test_vector512_width_rejects_short_columns(gpu_required):
    """A column whose prognostic levels are fewer than 16 has no Vector512 chunk (the reference
    would index below level 0): rejected with GRAL_EINVAL."""
    from gral_b200.prognostic import GralError
    dom = prep.small_domain(16, 14, seed=0)        # VertCellsFF 12
    sit = prep.Situation()
    with pytest.raises(GralError):
        solve_gpu(dom, [dom.params(sit, iterations=2, simd_width=16)], [prep.initial_fields(dom, sit)])


@pytest.mark.parametrize("model", [1, 2])
def test_post_diagnostic(gpu_required, layout, model):
    """post_diagnostic: DiagnosticFlowfield.Calculate (10 full-height pressure iterations) and the
    final vertical velocity of the columns outside the prognostic sub-domains, after the solve."""
    dom = prep.small_domain(20, 18, seed=15, n_buildings=3, subdomain_factor=1)
    assert (dom.static.advdom[2:-2, 2:-2] == 0).any()
    sits = [prep.Situation(direction_deg=d, speed_10m=3.0, z0=0.2, ustar=0.3) for d in (240.0, 40.0)]
    names = ("uk", "vk", "wk") + (("turb", "tdiss") if model == 2 else ())
    for fg, fc, sg, sc, tg, tc in run_pair(dom, sits, 4, model=model, post_diagnostic=1):
        np.testing.assert_array_equal(tg, tc)
        check_same(fg, fc, names)


def test_post_diagnostic_full_height_cube(gpu_required, layout):
    """The cube grid: NKK 162, so the diagnostic sweep covers 161 levels per column."""
    dom = prep.cube_domain()
    sit = prep.Situation(direction_deg=270.0, speed_10m=3.0, z0=0.2, ustar=0.3)
    for fg, fc, sg, sc, tg, tc in run_pair(dom, [sit], 2, post_diagnostic=1):
        check_same(fg, fc)
