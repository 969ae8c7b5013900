"""The library's discrete adjoint (``gral_prog_vjp_forward`` / ``gral_prog_vjp``) on the GPU,
through the C ABI, against the CPU references of the same unrolled iterations:

* the FP64 tape gradient of the oracle's twin (the same cotangents, the same map), relative L2
  difference of the VEG and initial-field gradients within 2e-3;
* FP64 central differences of the twin along 20 random directions of VEG (and of the initial
  fields) on a 32x32 grid over 20 iterations, every directional derivative within 1e-3 relative;
* checkpoint spacing: the gradient does not depend on it beyond float noise;
* rejection of the configurations it does not differentiate, and of a call out of order.

Differentiated configuration: turbulence model 1, parity width 8, no Frund rounding.
"""
import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.abi import GRAL_EINVAL, GRAL_ESTATE
from gral_b200.prognostic import GralError, PrognosticSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_vjp(dom, p, f, iterations, every, g):
    fg = f.copy()
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        s.vjp_forward(p, dom.static, fg, iterations, every)
        out = s.vjp(*(a.astype(np.float32) for a in g))
    return fg, out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_vjp_matches_the_fp64_tape_gradient(gpu_required):
    dom = prep.small_domain(16, 16, seed=3, with_veg=True)
    sit = prep.Situation(direction_deg=200.0, speed_10m=3.0)
    f = prep.initial_fields(dom, sit)
    n = 12
    p = dom.params(sit, model=1, iterations=n, quantise=0)
    x0 = (f.uk.astype(np.float64), f.vk.astype(np.float64), f.wk.astype(np.float64))
    veg = dom.static.veg.astype(np.float64)
    u, v, w = O.twin_forward(p, dom.static, f, x0, veg, n)
    idx, tgt = prep.probe_misfit(dom, prep.FieldArrays(u, v, w), n_probes=80, seed=4)
    _, g = prep.misfit_and_cotangent(idx, tgt, u, v, w)
    ref = O.twin_vjp(p, dom.static, f, x0, veg, n, g)
    fg, (d_veg, d_uk0, d_vk0, d_wk0, st) = gpu_vjp(dom, p, f, n, 5, g)
    # the forward is the solver's own (no rounding): it equals the float oracle bit for bit
    fo = f.copy()
    O.solve(p, dom.static, fo)
    np.testing.assert_array_equal(fg.uk, fo.uk)
    np.testing.assert_array_equal(fg.wk, fo.wk)
    # VEG enters the drag terms of the vegetation columns (veg_mask), at every level there
    cols = np.broadcast_to(dom.static.veg_mask[:, :, None] == 1, d_veg.shape)
    assert rel_l2(d_veg[cols], ref[3][cols]) <= 2e-3
    assert np.abs(d_veg[~cols]).max() == 0.0
    for a, b in ((d_uk0, ref[0]), (d_vk0, ref[1]), (d_wk0, ref[2])):
        assert rel_l2(a, b) <= 2e-3, rel_l2(a, b)
    assert st["iterations"] == n and st["checkpoint_every"] == 5


def test_vjp_matches_fp64_central_differences_32x32(gpu_required):
    dom = prep.adjoint_domain(32, n_buildings=3)
    sit = prep.Situation(direction_deg=235.0, speed_10m=2.0, z0=0.3)
    f = prep.initial_fields(dom, sit)
    n = 20
    p = dom.params(sit, model=1, iterations=n, quantise=0)
    x0 = (f.uk.astype(np.float64), f.vk.astype(np.float64), f.wk.astype(np.float64))
    veg = dom.static.veg.astype(np.float64)
    u, v, w = O.twin_forward(p, dom.static, f, x0, veg, n)
    idx, tgt = prep.probe_misfit(dom, prep.FieldArrays(u, v, w), n_probes=200, seed=5)
    _, g = prep.misfit_and_cotangent(idx, tgt, u, v, w)
    _, (d_veg, d_uk0, d_vk0, d_wk0, _) = gpu_vjp(dom, p, f, n, 20, g)

    def J(xx, vg):
        return prep.misfit_and_cotangent(idx, tgt, *O.twin_forward(p, dom.static, f, xx, vg, n))[0]

    rng = np.random.default_rng(21)
    mask = (veg > 0).astype(np.float64)
    errs = []
    for q in range(20):
        dv = rng.normal(size=veg.shape) * mask * 0.05
        du = rng.normal(size=f.uk.shape) * 0.01 * (np.abs(x0[0]) > 0) if q % 4 == 3 else 0.0 * x0[0]
        h = 1e-4
        fd = (J((x0[0] + h * du, x0[1], x0[2]), veg + h * dv) - J((x0[0] - h * du, x0[1], x0[2]), veg - h * dv)) / (2 * h)
        ad = float((d_veg.astype(np.float64) * dv).sum() + (d_uk0.astype(np.float64) * du).sum())
        errs.append(abs(fd - ad) / max(abs(fd), 1e-12))
    assert max(errs) <= 1e-3, errs


def test_vjp_does_not_depend_on_the_checkpoint_spacing(gpu_required):
    dom = prep.small_domain(16, 14, seed=5, with_veg=True)
    sit = prep.Situation(direction_deg=60.0, speed_10m=2.5)
    f = prep.initial_fields(dom, sit)
    n = 9
    p = dom.params(sit, model=1, iterations=n, quantise=0)
    fo = f.copy()
    O.solve(p, dom.static, fo)
    idx, tgt = prep.probe_misfit(dom, fo, n_probes=40, seed=6)
    _, g = prep.misfit_and_cotangent(idx, tgt, fo.uk, fo.vk, fo.wk)
    # 0: every iteration's states kept by the forward, nothing recomputed
    outs = [gpu_vjp(dom, p, f, n, k, g)[1] for k in (1, 4, 9, 0)]
    for o in outs[1:]:
        for a, b in zip(o[:4], outs[0][:4]):
            assert rel_l2(a, b) <= 1e-5
    assert outs[3][4]["ms_recompute"] < outs[1][4]["ms_recompute"]


def test_vjp_rejects_other_configurations_and_order(gpu_required):
    dom = prep.small_domain(16, 14, seed=0)
    sit = prep.Situation()
    f = prep.initial_fields(dom, sit, 2)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        g = np.zeros_like(f.uk)
        with pytest.raises(GralError) as e:
            s.vjp(g)
        assert e.value.code == GRAL_ESTATE
        for kw in (dict(model=2, quantise=0), dict(model=1, quantise=1), dict(model=1, quantise=0, simd_width=16)):
            p = dom.params(sit, iterations=3, **kw)
            with pytest.raises(GralError) as e:
                s.vjp_forward(p, dom.static, f.copy(), 3, 1)
            assert e.value.code == GRAL_EINVAL
        p = dom.params(sit, iterations=3, model=1, quantise=0)
        with pytest.raises(GralError) as e:   # a negative checkpoint spacing
            s.vjp_forward(p, dom.static, f.copy(), 3, -1)
        assert e.value.code == GRAL_EINVAL
