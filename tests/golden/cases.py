"""Golden cases of the prognostic solve (turbulence models 0, 1 and 2; model 1 with the
Vector<float> width 8 and the Vector512 width 16).

Inputs are rebuilt from ``gral_b200.prep`` with the seeds stated here, so only outputs are stored:
``<name>.npz`` (fields, DeltaUMax trace, statistics) for the small grids and SHA-256 digests in
``checksums.json`` for the full-size grids (the 100x100x162 cube and the 400x400x63 city, also at
the benchmark lengths of 100 and 500 iterations with the reference's stop rule, and eight
situations of the 144-situation weather set).  The
outputs were written by ``make_golden.py`` from the CPU oracle; ``MANIFEST.json`` records the
oracle sources' digests and the reference version the oracle restates.
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Dict, List, Tuple

import numpy as np

from gral_b200 import prep

HERE = os.path.dirname(os.path.abspath(__file__))

# name: (domain builder, domain kwargs, situations, model, iterations, params kwargs, stored as)
CASES: Dict[str, tuple] = {
    "m1_small_s0": ("small", dict(nii=16, njj=14, seed=0), [(250.0, 3.0, 0.2, 0.3)], 1, 6, {}, "npz"),
    "m1_small_s1": ("small", dict(nii=16, njj=14, seed=1), [(280.0, 3.0, 0.2, 0.3)], 1, 9, {}, "npz"),
    "m1_dirs_s2": ("small", dict(nii=18, njj=15, seed=2, n_buildings=4),
                   [(15.0, 2.0, 0.3, 0.25), (135.0, 4.0, 0.3, 0.25), (290.0, 1.0, 0.3, 0.25)], 1, 7, {}, "npz"),
    "m1_veg_s3": ("small", dict(nii=16, njj=16, seed=3, with_veg=True), [(200.0, 3.0, 0.2, 0.3)], 1, 6, {}, "npz"),
    "m1_conv_s4": ("small", dict(nii=14, njj=12, seed=4, n_buildings=2), [(260.0, 3.0, 0.2, 0.3)], 1, 400,
                   dict(iter_min=100, conv_threshold=0.05), "npz"),
    "m1_noquant_s5": ("small", dict(nii=16, njj=14, seed=5), [(45.0, 2.0, 0.2, 0.3)], 1, 5, dict(quantise=0), "npz"),
    "m2_small_s6": ("small", dict(nii=16, njj=14, seed=6, obukhov=-80.0), [(230.0, 3.0, 0.2, 0.3)], 2, 8, {}, "npz"),
    "m2_dirs_s7": ("small", dict(nii=18, njj=15, seed=7, n_buildings=4, obukhov=200.0),
                   [(20.0, 2.0, 0.3, 0.25), (140.0, 4.0, 0.3, 0.25), (300.0, 1.5, 0.3, 0.25)], 2, 5, {}, "npz"),
    "m2_veg_s8": ("small", dict(nii=16, njj=16, seed=8, with_veg=True), [(110.0, 3.0, 0.2, 0.3)], 2, 5, {}, "npz"),
    "m0_small_s9": ("small", dict(nii=16, njj=14, seed=9), [(320.0, 2.5, 0.2, 0.3)], 0, 4, {}, "npz"),
    "m1w16_small_s12": ("small", dict(nii=16, njj=14, seed=12, vert_cells_ff=20), [(250.0, 3.0, 0.2, 0.3)], 1, 6,
                        dict(simd_width=16), "npz"),
    "m1w16_veg_s13": ("small", dict(nii=16, njj=16, seed=13, vert_cells_ff=20, with_veg=True),
                      [(160.0, 3.0, 0.2, 0.3), (20.0, 2.0, 0.2, 0.3)], 1, 5, dict(simd_width=16), "npz"),
    "m1_diag_s15": ("small", dict(nii=20, njj=18, seed=15, n_buildings=3, subdomain_factor=1),
                    [(240.0, 3.0, 0.2, 0.3)], 1, 4, dict(post_diagnostic=1), "npz"),
    "m1_cube_100": ("cube", dict(), [(270.0, 3.0, 0.2, 0.3)], 1, 3, {}, "sha"),
    "m1_diag_cube_100": ("cube", dict(), [(270.0, 3.0, 0.2, 0.3)], 1, 3, dict(post_diagnostic=1), "sha"),
    "m1w16_cube_100": ("cube", dict(), [(270.0, 3.0, 0.2, 0.3)], 1, 3, dict(simd_width=16), "sha"),
    "m1_city_400": ("city", dict(), [(225.0, 2.0, 0.5, 0.3)], 1, 2, {}, "sha"),
    # the benchmark configurations at their own length, with the reference's stop rule (_delta <
    # 0.012 tested every 100 iterations from IterationStepsMin = 100 on)
    "m1_cube_full": ("cube", dict(), [(270.0, 3.0, 0.2, 0.3)], 1, 100, {}, "sha"),
    "m1_cube_conv500": ("cube", dict(), [(270.0, 3.0, 0.2, 0.3)], 1, 500, dict(iter_min=100), "sha"),
    "m1_city_full": ("city", dict(), [(225.0, 2.0, 0.5, 0.3)], 1, 500, dict(iter_min=100), "sha"),
    # eight situations of the 144-situation weather set on the production grid (all four speeds,
    # directions 0..350 deg, seeded stability), each stopping at its own iteration
    "m1_city_weather8": ("city", dict(), "weather:1,22,43,64,87,106,125,140", 1, 500, dict(iter_min=100), "sha"),
}

# cases whose oracle run takes minutes (500 iterations on the production grid): their digests are
# written by make_golden.py and checked against the GPU only; the CPU suite re-runs the others
LONG = {"m1_cube_conv500", "m1_city_full", "m1_city_weather8"}

FIELDS = ("uk", "vk", "wk", "turb", "tdiss")
STAT_KEYS = ("iterations", "iteration_loops", "converged", "convergence_problem", "delta_first",
             "delta_finish", "delta_history", "uk_unrealistic", "vk_unrealistic", "wk_unrealistic",
             "geschw_max", "topwind", "dtime", "frund", "last_delta_umax")


def domain(name: str):
    kind, kw = CASES[name][0], CASES[name][1]
    if kind == "small":
        return prep.small_domain(**kw)
    if kind == "cube":
        return prep.cube_domain(**kw)
    if kind == "city":
        return prep.city_domain(**kw)
    raise KeyError(kind)


def situations(name: str) -> List[prep.Situation]:
    """The situations of a case: (direction, speed, z0, u*) tuples, or "weather:<indices>" naming
    members of prep.weather_situations()."""
    sits = CASES[name][2]
    if isinstance(sits, str):
        pool = prep.weather_situations()
        return [pool[int(q)] for q in sits.split(":", 1)[1].split(",")]
    return [prep.Situation(direction_deg=d, speed_10m=v, z0=z0, ustar=us) for d, v, z0, us in sits]


def build(name: str):
    """(domain, [params], [initial fields]) of a case."""
    _, _, sits, model, iters, pkw, _ = CASES[name]
    dom = domain(name)
    ps, fs = [], []
    for sit in situations(name):
        ps.append(dom.params(sit, model=model, iterations=iters, **pkw))
        fs.append(prep.initial_fields(dom, sit, model))
    return dom, ps, fs


def storage(name: str) -> str:
    return CASES[name][6]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def stats_subset(st: dict) -> dict:
    return {k: st[k] for k in STAT_KEYS}


def load_npz(name: str) -> Tuple[List[dict], List[dict], List[np.ndarray]]:
    """Stored outputs of an npz case: per situation the fields dict, the stats and the trace."""
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    stats = json.loads(str(z["stats"]))
    n = len(stats)
    fields = [{f: z[f"{f}_{b}"] for f in FIELDS if f"{f}_{b}" in z.files} for b in range(n)]
    traces = [z[f"trace_{b}"] for b in range(n)]
    return fields, stats, traces


def load_sha() -> dict:
    with open(os.path.join(HERE, "checksums.json")) as fh:
        return json.load(fh)


def outputs_sha(fields_list, stats_list, traces) -> list:
    out = []
    for f, st, tr in zip(fields_list, stats_list, traces):
        d = {name: digest(getattr(f, name)) for name in FIELDS if getattr(f, name) is not None}
        d["trace"] = digest(tr)
        d["stats"] = stats_subset(st)
        out.append(d)
    return out
