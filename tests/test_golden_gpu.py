"""The CUDA solver (through the C ABI) against the committed golden outputs, in both kernel
families (slab and interleaved layouts), bit for bit: fields, DeltaUMax traces and statistics."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import cases as G  # noqa: E402
from gral_b200.prognostic import PrognosticSolver  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["slab", "interleaved"])
def layout(request, monkeypatch):
    monkeypatch.setenv("GRAL_PROG_LAYOUT", request.param)
    return request.param


def run_gpu(name):
    dom, ps, fs = G.build(name)
    traces = [np.zeros(max(p["iteration_steps_max"], 1), np.float32) for p in ps]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(ps)) as s:
        stats = s.calculate_batch(ps, dom.static, fs, traces)
    return fs, stats, traces


@pytest.mark.parametrize("name", list(G.CASES))
def test_gpu_matches_golden(gpu_required, layout, name):
    fs, stats, traces = run_gpu(name)
    if G.storage(name) == "sha":
        assert G.outputs_sha(fs, stats, traces) == G.load_sha()[name]
        return
    gf, gs, gt = G.load_npz(name)
    for b in range(len(stats)):
        for fld, want in gf[b].items():
            np.testing.assert_array_equal(getattr(fs[b], fld), want, err_msg=f"{name}[{b}].{fld}")
        np.testing.assert_array_equal(traces[b], gt[b])
        assert G.stats_subset(stats[b]) == gs[b]
