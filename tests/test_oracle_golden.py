"""The CPU oracle against the committed golden outputs (tests/golden), bit for bit.

The golden files were written by tests/golden/make_golden.py from this oracle; the C# reference
cannot run here and ships no test vectors for the prognostic solve, so parity with the reference
itself is unpinned.  These tests pin the oracle against regressions of its own sources and of the
input builders in gral_b200.prep, for every turbulence model and both storage kinds (full arrays
for the small grids, SHA-256 digests for the 100x100x162 cube and the 400x400x63 city grid).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import cases as G  # noqa: E402
from oracle import oracle as O  # noqa: E402


def run_oracle(name):
    dom, ps, fs = G.build(name)
    stats, traces = [], []
    for p, f in zip(ps, fs):
        tr = np.zeros(max(p["iteration_steps_max"], 1), np.float32)
        stats.append(O.solve(p, dom.static, f, tr))
        traces.append(tr)
    return fs, stats, traces


@pytest.mark.parametrize("name", [n for n in G.CASES if G.storage(n) == "npz"])
def test_oracle_matches_golden_arrays(name):
    fs, stats, traces = run_oracle(name)
    gf, gs, gt = G.load_npz(name)
    assert len(gs) == len(stats)
    for b in range(len(stats)):
        for fld, want in gf[b].items():
            np.testing.assert_array_equal(getattr(fs[b], fld), want, err_msg=f"{name}[{b}].{fld}")
        np.testing.assert_array_equal(traces[b], gt[b])
        assert G.stats_subset(stats[b]) == gs[b]


@pytest.mark.parametrize("name", [n for n in G.CASES if G.storage(n) == "sha" and n not in G.LONG])
def test_oracle_matches_golden_digests(name):
    fs, stats, traces = run_oracle(name)
    assert G.outputs_sha(fs, stats, traces) == G.load_sha()[name]


def test_golden_covers_every_model_and_full_size_geometry():
    models = {G.CASES[n][3] for n in G.CASES}
    assert models == {0, 1, 2}
    assert {"m1_cube_100", "m1_city_400"} <= set(G.load_sha())
    assert set(G.LONG) | {"m1_cube_full"} <= set(G.load_sha())
    for name in G.CASES:
        if G.storage(name) == "npz":
            assert os.path.exists(os.path.join(G.HERE, f"{name}.npz")), name


def test_golden_convergence_case_stops_at_cadence():
    """The convergence case stops at a multiple of the 100-iteration cadence before its maximum,
    with one residual per cadence point."""
    _, gs, _ = G.load_npz("m1_conv_s4")
    st = gs[0]
    assert st["converged"] == 1
    assert st["iterations"] % 100 == 0 and st["iterations"] < 400
    assert len(st["delta_history"]) == st["iterations"] // 100


def test_golden_benchmark_lengths_and_stop_rule():
    """The benchmark configurations at their own length: the 100x100 cube for 100 iterations and
    for up to 500 with the reference's stop rule (0.012, tested every 100 iterations), the
    production grid for 500, and eight situations of the weather set; the stop rule's decisions
    are part of the digests (iterations, converged flag, residual history at 100, 200, ...)."""
    sha = G.load_sha()
    assert [x["stats"]["iterations"] for x in sha["m1_cube_full"]] == [100]
    for name in ("m1_cube_conv500", "m1_city_full", "m1_city_weather8"):
        for x in sha[name]:
            st = x["stats"]
            assert len(st["delta_history"]) == st["iterations"] // 100
            assert st["converged"] == 1 or st["iterations"] == 500
    assert len(sha["m1_city_weather8"]) == 8
