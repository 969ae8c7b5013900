"""A batch spread over several devices through the library (``gral_prog_solve_batch_devices``).

Weather situations are independent, so a batch shards by situation with no exchange between
devices: each listed device takes a contiguous shard in a context of its own.  On a node with one
GPU the device is listed twice, which runs two contexts side by side on it; every situation must
come out bit-identical to a single-context solve of the whole batch, with the same iteration
counts and per-situation statistics.
"""
import numpy as np
import pytest

from gral_b200 import abi, prep
from gral_b200.prognostic import PrognosticSolver, solve_batch_devices

pytestmark = pytest.mark.gpu


def test_batch_over_devices_matches_one_context(gpu_required):
    import torch
    ndev = torch.cuda.device_count()
    devices = list(range(ndev)) if ndev > 1 else [0, 0]
    dom = prep.small_domain(20, 18, seed=5, n_buildings=3, with_veg=True)
    sits = [prep.random_situation(900 + q) for q in range(5)]
    ps = [dom.params(x, model=1, iterations=7) for x in sits]
    f0 = [prep.initial_fields(dom, x) for x in sits]
    one = [f.copy() for f in f0]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(sits)) as s:
        st1 = s.calculate_batch(ps, dom.static, one)
    got = [f.copy() for f in f0]
    st2, rc = solve_batch_devices(devices, ps, dom.static, got)
    assert rc == abi.GRAL_OK
    for b in range(len(sits)):
        for name in ("uk", "vk", "wk"):
            assert np.array_equal(getattr(got[b], name), getattr(one[b], name)), (b, name)
        assert st2[b]["iterations"] == st1[b]["iterations"] == 7
        assert st2[b]["delta_finish"] == st1[b]["delta_finish"]


def test_batch_over_devices_rejects_a_bad_ordinal(gpu_required):
    dom = prep.small_domain(16, 14, seed=0)
    sit = prep.Situation()
    ps = [dom.params(sit, iterations=2)] * 2
    fs = [prep.initial_fields(dom, sit) for _ in range(2)]
    _, rc = solve_batch_devices([0, 4096], ps, dom.static, fs)
    assert rc == abi.GRAL_EINVAL
