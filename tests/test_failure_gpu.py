"""Failure paths and edge cases of the GPU solver, with no GPU fault involved.

* A wavefront wait that runs out: every device-side spin wait is bounded; with the bound set to
  1 ns (GRAL_PROG_WAIT_NS) the first wait that does not succeed at once gives up, sets the error
  word and returns, the solve reports GRAL_ETIMEDOUT, and the same process then solves normally.
* Non-finite input without quantisation: the post-check reports GRAL_ENONFINITE.
* A grid without any prognostic sub-domain, and a batch whose situations meet the convergence
  test at different iterations (per-situation stop): both against the oracle.
"""
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


def test_wait_timeout_is_reported_and_recoverable(gpu_required, monkeypatch, layout):
    dom = prep.small_domain(60, 60, seed=22, n_buildings=6)
    sit = prep.Situation(direction_deg=230.0, speed_10m=3.0)
    p = dom.params(sit, model=1, iterations=4)
    monkeypatch.setenv("GRAL_PROG_WAIT_NS", "1")
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        with pytest.raises(GralError) as e:
            s.calculate(p, dom.static, prep.initial_fields(dom, sit))
        assert e.value.code == abi.GRAL_ETIMEDOUT
        monkeypatch.delenv("GRAL_PROG_WAIT_NS")
        f = prep.initial_fields(dom, sit)
        fc = f.copy()
        st = s.calculate(p, dom.static, f)            # same context, fresh load: normal result
    O.solve(p, dom.static, fc)
    assert st["iterations"] == 4
    for name in ("uk", "vk", "wk"):
        np.testing.assert_array_equal(getattr(f, name), getattr(fc, name))


def test_nonfinite_input_is_reported(gpu_required, layout):
    dom = prep.small_domain(16, 14, seed=23)
    sit = prep.Situation(direction_deg=200.0)
    p = dom.params(sit, model=1, iterations=3, quantise=0)
    f = prep.initial_fields(dom, sit)
    i, j = np.argwhere(dom.static.advdom[2:-2, 2:-2] == 1)[5] + 2
    f.uk[i, j, dom.static.kkart[i, j] + 3] = np.nan
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        with pytest.raises(GralError) as e:
            s.calculate(p, dom.static, f)
    assert e.value.code == abi.GRAL_ENONFINITE


def test_no_prognostic_subdomain(gpu_required, layout):
    dom = prep.small_domain(16, 14, seed=21)
    dom.static.advdom[:] = 0
    sit = prep.Situation(direction_deg=250.0)
    p = dom.params(sit, model=1, iterations=3)
    f = prep.initial_fields(dom, sit)
    fc = f.copy()
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        st = s.calculate(p, dom.static, f)
    sc = O.solve(p, dom.static, fc)
    assert st["iterations"] == sc["iterations"] == 3
    for name in ("uk", "vk", "wk"):
        np.testing.assert_array_equal(getattr(f, name), getattr(fc, name))


def test_batch_stops_each_situation_at_its_own_iteration(gpu_required, layout):
    """Three situations, thresholds 0.5 / 0.05 / 0: they leave the loop at iterations 200, 300
    (converged) and 300 (maximum, not converged), each with the oracle's fields and history."""
    dom = prep.small_domain(14, 12, seed=4, n_buildings=2)
    sit = prep.Situation(direction_deg=260.0)
    ps = [dom.params(sit, model=1, iterations=300, iter_min=100, conv_threshold=t) for t in (0.5, 0.05, 0.0)]
    fs = [prep.initial_fields(dom, sit) for _ in ps]
    fcs = [f.copy() for f in fs]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=3) as s:
        sts = s.calculate_batch(ps, dom.static, fs)
    assert [x["iterations"] for x in sts] == [200, 300, 300]
    assert [x["converged"] for x in sts] == [1, 1, 0]
    for b in range(3):
        sc = O.solve(ps[b], dom.static, fcs[b])
        assert sts[b]["iterations"] == sc["iterations"]
        assert sts[b]["delta_history"] == sc["delta_history"]
        for name in ("uk", "vk", "wk"):
            np.testing.assert_array_equal(getattr(fs[b], name), getattr(fcs[b], name))
