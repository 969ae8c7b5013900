"""The allocation-free speed check (``gral_prog_check_speeds_noalloc``) against the solver's own.

The entry point serves callers that keep a solved flow field on the GPU and cannot call cudaMalloc
when they check it (device memory committed to their own pool, or no device-wide synchronisation
allowed while other streams run).  It runs the post-solve unrealistic-speed check on caller-owned
device arrays with its scratch in a fixed static device array.  Here its counts must equal the
ones ``gral_prog_solve_batch`` reports for the same solved fields, on two calls in a row (the
second call must not see the first call's partial counts), and oversized or host inputs must be
rejected before any GPU work.  The device copies of the inputs are made with torch by the test;
the entry point itself allocates nothing.

This file is collected last on purpose, so that a run stopping at its first failure has already
run every other test.
"""

import numpy as np
import pytest

from gral_b200 import prep
from gral_b200.abi import GRAL_EINVAL, GRAL_ETOOLARGE, GRAL_NOALLOC_MAX_ROWS
from gral_b200.prognostic import GralError, PrognosticSolver, check_speeds_noalloc, lib

pytestmark = pytest.mark.gpu

# (direction, 10 m speed): strong enough that levels below KKART+vert_cells_ff exceed 55 m/s,
# in U for the first case and in V for the second, so the two calls give different counts
CASES = [(250.0, 60.0), (160.0, 48.0)]


def solved_case(direction, speed):
    dom = prep.small_domain(16, 14, seed=11)
    sit = prep.Situation(direction_deg=direction, speed_10m=speed)
    f = prep.initial_fields(dom, sit, 1)
    p = dom.params(sit, model=1, iterations=3)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        st = s.calculate(p, dom.static, f)
    return dom, f, st


def test_check_speeds_noalloc_matches_solver(gpu_required):
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    seen = []
    for direction, speed in CASES:
        dom, f, st = solved_case(direction, speed)
        d_uk, d_vk, d_wk = (torch.from_numpy(a).to(dev) for a in (f.uk, f.vk, f.wk))
        d_adv = torch.from_numpy(dom.static.advdom).to(dev)
        d_kk = torch.from_numpy(dom.static.kkart).to(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        torch.cuda.synchronize(dev)
        got = check_speeds_noalloc(dom.nii, dom.njj, dom.nkk, dom.vert_cells_ff, st["geschw_max"],
                                   d_uk.data_ptr(), d_vk.data_ptr(), d_wk.data_ptr(), d_adv.data_ptr(),
                                   d_kk.data_ptr(), stream)
        want = (st["uk_unrealistic"], st["vk_unrealistic"], st["wk_unrealistic"], 0)
        assert got == want, (direction, speed)
        seen.append(got)
    assert seen[0] != seen[1]
    assert seen[0][0] > 0 and seen[1][1] > 0


def test_check_speeds_noalloc_rejects(gpu_required):
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    n = 8
    d = torch.zeros((n + 2) * (n + 2) * (n + 2), dtype=torch.float32, device=dev)
    a = torch.zeros((n + 2) * (n + 2), dtype=torch.uint8, device=dev)
    k = torch.zeros((n + 2) * (n + 2), dtype=torch.int16, device=dev)
    with pytest.raises(GralError) as e:
        check_speeds_noalloc(GRAL_NOALLOC_MAX_ROWS + 1, n, n, 4, 1.0, d.data_ptr(), d.data_ptr(),
                             d.data_ptr(), a.data_ptr(), k.data_ptr())
    assert e.value.code == GRAL_ETOOLARGE
    host = np.zeros((n + 2) ** 3, np.float32)
    with pytest.raises(GralError) as e:
        check_speeds_noalloc(n, n, n, 4, 1.0, host.ctypes.data, d.data_ptr(), d.data_ptr(), a.data_ptr(),
                             k.data_ptr())
    assert e.value.code == GRAL_EINVAL
    # a valid call on the same device still works after the rejected ones
    assert check_speeds_noalloc(n, n, n, 4, 1.0, d.data_ptr(), d.data_ptr(), d.data_ptr(), a.data_ptr(),
                                k.data_ptr()) == (0, 0, 0, 0)
    assert lib().gral_prog_check_speeds_noalloc(n, n, n, 4, 1.0, d.data_ptr(), d.data_ptr(), d.data_ptr(),
                                                a.data_ptr(), k.data_ptr(), None, None) == GRAL_EINVAL


def test_check_speeds_noalloc_rejects_other_device(gpu_required):
    """Device memory of another GPU is refused on the host before any launch (needs two GPUs)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU to hold the foreign arrays")
    n = 8
    torch.cuda.set_device(0)
    d0 = torch.zeros((n + 2) ** 3, dtype=torch.float32, device="cuda:0")
    a0 = torch.zeros((n + 2) ** 2, dtype=torch.uint8, device="cuda:0")
    k0 = torch.zeros((n + 2) ** 2, dtype=torch.int16, device="cuda:0")
    d1 = torch.zeros((n + 2) ** 3, dtype=torch.float32, device="cuda:1")
    with pytest.raises(GralError) as e:
        check_speeds_noalloc(n, n, n, 4, 1.0, d1.data_ptr(), d0.data_ptr(), d0.data_ptr(), a0.data_ptr(),
                             k0.data_ptr())
    assert e.value.code == GRAL_EINVAL
