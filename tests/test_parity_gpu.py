"""GPU parity: the CUDA solver (through the C ABI) against the CPU oracle on the same inputs.

Both implement the reference's deterministic float32 evaluation order, so the expected difference
is zero; the asserted bound is the north-star tolerance max|dU|/max|U| <= 1e-4 with the
iteration count and convergence decisions compared exactly.
"""
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


def run_both(dom, sit, iterations, model=1, **kw):
    p = dom.params(sit, model=model, iterations=iterations, **kw)
    f_gpu = prep.initial_fields(dom, sit, model)
    f_cpu = f_gpu.copy()
    tr_g = np.zeros(max(iterations, 1), np.float32)
    tr_c = np.zeros(max(iterations, 1), np.float32)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        sg = s.calculate(p, dom.static, f_gpu, trace=tr_g)
    sc = O.solve(p, dom.static, f_cpu, trace=tr_c)
    return f_gpu, f_cpu, sg, sc, tr_g, tr_c


@pytest.mark.parametrize("iterations", [1, 2, 4, 9])
@pytest.mark.parametrize("seed", [0, 1])
def test_model1_small(gpu_required, seed, iterations):
    dom = prep.small_domain(16, 14, seed=seed)
    sit = prep.Situation(direction_deg=250.0 + 30 * seed, speed_10m=3.0, z0=0.2, ustar=0.3)
    fg, fc, sg, sc, tg, tc = run_both(dom, sit, iterations)
    assert sg["iterations"] == sc["iterations"] == iterations
    np.testing.assert_array_equal(tg, tc)
    for name in ("uk", "vk", "wk"):
        a, b = getattr(fg, name), getattr(fc, name)
        assert rel_err(a, b) <= TOL, name
        assert np.array_equal(a, b), f"{name} not bit-identical"
