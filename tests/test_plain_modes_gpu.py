"""Every schedule of the slab family's model-1 sweeps gives the oracle's result bit for bit.

The slab family (one or a few situations) runs the pressure and the U, V, W sweeps either on the
diagonal-claim wavefront (mode 0: one warp per column task, every hand-off through a global flag)
or on a strip schedule (mode 1+v: a block per strip of sweep rows, hand-offs inside the strip
through shared-memory progress counters; the last mode runs pressure, velocity correction,
averages and U as one launch whose claims alternate pressure strips and U strips).  The autotuner may keep any of them, so each is forced
in turn (GRAL_PROG_PLAIN_MODE) over six iterations, which cover all four sweep directions, on a
grid whose row count is not a multiple of any strip height, with buildings and vegetation, for
one situation and for three (strips of different situations claimed from one counter), at both
parity widths.  Fields and DeltaUMax traces must equal the oracle's.
"""
import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.prognostic import PrognosticSolver
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ITERS = 6


@pytest.mark.parametrize("n_sit,simd", [(1, 8), (3, 8), (1, 16)])
def test_every_plain_mode_matches_oracle(gpu_required, monkeypatch, n_sit, simd):
    dom = prep.small_domain(23, 19, seed=11, n_buildings=4, with_veg=True, vert_cells_ff=20)
    sits = [prep.random_situation(500 + q) for q in range(n_sit)]
    ps = [dom.params(x, model=1, iterations=ITERS, simd_width=simd) for x in sits]
    f0 = [prep.initial_fields(dom, x, 1) for x in sits]
    want, want_tr = [], []
    for b in range(n_sit):
        fc = f0[b].copy()
        tc = np.zeros(ITERS, np.float32)
        O.solve(ps[b], dom.static, fc, tc)
        want.append(fc)
        want_tr.append(tc)
    monkeypatch.setenv("GRAL_PROG_LAYOUT", "slab")
    seen = []
    for mode in range(16):
        monkeypatch.setenv("GRAL_PROG_PLAIN_MODE", str(mode))
        fg = [f.copy() for f in f0]
        tg = [np.zeros(ITERS, np.float32) for _ in range(n_sit)]
        with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=n_sit) as s:
            st = s.calculate_batch(ps, dom.static, fg, tg)
        if st[0]["launch_variant"] != mode:      # past the last mode: the request is ignored
            break
        seen.append(mode)
        for b in range(n_sit):
            assert st[b]["iterations"] == ITERS
            for name in ("uk", "vk", "wk"):
                assert np.array_equal(getattr(fg[b], name), getattr(want[b], name)), (mode, b, name)
            assert np.array_equal(tg[b], want_tr[b]), (mode, b, "DeltaUMax trace")
    # the diagonal-claim wavefront, four strip variants and the fused strips
    assert len(seen) >= 6, seen
