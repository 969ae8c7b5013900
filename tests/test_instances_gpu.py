"""Independent situations on grids of different sizes solved side by side
(``gral_prog_solve_instances``, the uneven-domain batch: hills and buildings, random inflow).

Every instance must come out bit-identical to the oracle and to a single ``gral_prog_solve`` of
the same inputs, with the same iteration counts, whatever the number of instances running at
once; an instance with a non-finite field reports GRAL_ENONFINITE in its own status while the
others succeed.
"""
import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.prognostic import PrognosticSolver, solve_instances
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [(24, 20, 2.0, 8), (40, 36, 3.0, 10), (32, 44, 2.5, 12), (48, 28, 4.0, 9), (20, 20, 2.0, 8),
         (36, 36, 3.5, 11)]


def instances(sizes, iterations, seed0=0):
    doms, ps, fs = [], [], []
    for q, (ni, nj, dx, vc) in enumerate(sizes):
        d = prep.hilly_domain(ni, nj, dx, vc, seed=seed0 + q)
        sit = prep.random_situation(seed0 + q)
        doms.append(d)
        ps.append(d.params(sit, model=1, iterations=iterations))
        fs.append(prep.initial_fields(d, sit))
    return doms, ps, fs


def assert_same(a, b):
    for name in ("uk", "vk", "wk"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)


def test_instances_match_oracle(gpu_required):
    doms, ps, fs = instances(SIZES, 12)
    got = [f.copy() for f in fs]
    stats, status, rc = solve_instances(ps, [d.static for d in doms], got, max_concurrent=3)
    assert rc == abi.GRAL_OK and status == [abi.GRAL_OK] * len(SIZES)
    for b, d in enumerate(doms):
        want = fs[b].copy()
        st = O.solve(ps[b], d.static, want)
        assert_same(got[b], want)
        assert stats[b]["iterations"] == st["iterations"] == 12


@pytest.mark.parametrize("concurrent", [1, 4])
def test_instances_match_single_solves(gpu_required, concurrent):
    sizes = [(128, 112, 2.0, 20), (160, 128, 3.0, 24), (96, 144, 4.0, 20), (192, 176, 2.5, 30)]
    doms, ps, fs = instances(sizes, 30, seed0=20)
    got = [f.copy() for f in fs]
    stats, status, rc = solve_instances(ps, [d.static for d in doms], got, max_concurrent=concurrent)
    assert rc == abi.GRAL_OK, status
    for b, d in enumerate(doms):
        one = fs[b].copy()
        with PrognosticSolver(d.nii, d.njj, d.nkk, d.kadvmax) as s:
            st = s.calculate(ps[b], d.static, one)
        assert_same(got[b], one)
        assert stats[b]["iterations"] == st["iterations"]
        assert stats[b]["delta_finish"] == st["delta_finish"]


def test_instance_failure_is_its_own(gpu_required):
    doms, ps, fs = instances(SIZES[:4], 6, seed0=40)
    bad = 2
    d = doms[bad]
    i, j = np.argwhere(d.static.advdom[2:-2, 2:-2] == 1)[7] + 2
    fs[bad].uk[i, j, d.static.kkart[i, j] + 2] = np.nan
    stats, status, rc = solve_instances(ps, [x.static for x in doms], fs, max_concurrent=2)
    assert status[bad] == abi.GRAL_ENONFINITE and rc == abi.GRAL_ENONFINITE
    assert [s for b, s in enumerate(status) if b != bad] == [abi.GRAL_OK] * 3


def test_instances_queue_and_memory_budget(gpu_required):
    """More instances than slots: each slot takes the next largest instance left when its own is
    done, in buffers sized by its first (larger) one.  An HBM budget of about twice the largest
    instance's footprint admits fewer slots than max_concurrent; results stay bit-identical."""
    sizes = SIZES + [(28, 24, 2.0, 9), (44, 40, 3.0, 12), (22, 30, 2.5, 8), (34, 26, 4.0, 10)]
    doms, ps, fs = instances(sizes, 8, seed0=60)
    want = []
    for b, d in enumerate(doms):
        w = fs[b].copy()
        O.solve(ps[b], d.static, w)
        want.append(w)
    for k, budget in ((4, 0), (8, 48 << 20)):
        got = [f.copy() for f in fs]
        stats, status, rc = solve_instances(ps, [d.static for d in doms], got, max_concurrent=k, hbm_bytes=budget)
        assert rc == abi.GRAL_OK and status == [abi.GRAL_OK] * len(sizes), status
        for b in range(len(sizes)):
            assert_same(got[b], want[b])
            assert stats[b]["iterations"] == 8

