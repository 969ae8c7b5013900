"""Every launch variant of the batched (interleaved) family gives the oracle's fields bit for bit.

The autotuner times the variants on live iterations and keeps the fastest, so any of them can
carry a production solve: warps per block and resident blocks per SM, and the group-set launch
modes (all groups, two, one per launch).  Each is forced in turn (GRAL_PROG_BATCH_VARIANT) on a
batch of three groups of situations (32, 32 and 6 situations) with vegetation, for models 0, 1
and 2.
"""
import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.prognostic import PrognosticSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_SITUATIONS = 70


@pytest.mark.parametrize("model", [0, 1, 2])
def test_every_launch_variant_matches_oracle(gpu_required, monkeypatch, model):
    dom = prep.small_domain(22, 18, seed=9, n_buildings=4, with_veg=True)
    sits = [prep.random_situation(300 + q) for q in range(N_SITUATIONS)]
    ps = [dom.params(x, model=model, iterations=5) for x in sits]
    f0 = [prep.initial_fields(dom, x, model) for x in sits]
    want = []
    for b in range(N_SITUATIONS):
        fc = f0[b].copy()
        O.solve(ps[b], dom.static, fc)
        want.append(fc)
    names = ("uk", "vk", "wk") + (("turb", "tdiss") if model == 2 else ())
    monkeypatch.setenv("GRAL_PROG_LAYOUT", "interleaved")
    seen = []
    for v in range(64):
        monkeypatch.setenv("GRAL_PROG_BATCH_VARIANT", str(v))
        fg = [f.copy() for f in f0]
        with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=N_SITUATIONS) as s:
            st = s.calculate_batch(ps, dom.static, fg)
        if st[0]["launch_variant"] != v:      # past the last variant: the request is ignored
            break
        seen.append(v)
        for b in range(N_SITUATIONS):
            assert st[b]["iterations"] == 5
            for name in names:
                assert np.array_equal(getattr(fg[b], name), getattr(want[b], name)), (v, b, name)
    # every kernel variant in each of the three group-set modes (at least four kernel variants)
    assert len(seen) >= 12 and len(seen) % 3 == 0
