"""Write the golden outputs of ``cases.py`` from the CPU oracle.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py m1_small_s0
    GRAL_REFERENCE_SRC=<GRAL checkout>/src python tests/golden/make_golden.py   # also hash the reference

Situations run in parallel worker processes (GOLDEN_WORKERS, default: every CPU), each one the
oracle's serial deterministic solve; the 500-iteration production-grid cases take about 7 minutes
of one core per situation.

The oracle is the deterministic restatement of GRAL's prognostic solve under ``oracle/``; the
C# reference cannot run in this environment, so these files pin the oracle (and through it the
GPU path) against regressions, not against the reference itself.  The manifest records the
oracle sources' SHA-256 and, when the reference tree is readable here, the digests of the
reference files the oracle restates.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

# source directory of the GRAL checkout the oracle restates (its `src/` folder); taken from the
# environment so that no machine path is built in; without it the previous manifest's reference
# digests are kept
REFERENCE_TREE = os.environ.get("GRAL_REFERENCE_SRC", "")
REFERENCE_FILES = ["PrognosticFlowfield.cs", "U-prognostic-microscale_0.cs", "U-prognostic-microscale_1.cs",
                   "U-prognostic-microscale_2.cs", "V-prognostic-microscale_0.cs", "V-prognostic-microscale_1.cs",
                   "V-prognostic-microscale_2.cs", "W-prognostic-microscale_0.cs", "W-prognostic-microscale_1.cs",
                   "W-prognostic-microscale_2.cs", "TKE-prognostic-microscale.cs", "ProgramFunctions.cs"]


def sha_file(p: str) -> str:
    with open(p, "rb") as fh:
        return hashlib.sha256(fh.read()).hexdigest()


def _solve_one(job):
    """One situation of a case in a worker process: (fields, stats, trace)."""
    name, b = job
    dom, ps, fs = G.build(name)
    tr = np.zeros(max(ps[b]["iteration_steps_max"], 1), np.float32)
    st = O.solve(ps[b], dom.static, fs[b], tr)
    return fs[b], st, tr


def run_cases(names, workers: int):
    """Outputs of every situation of every case; situations run in `workers` processes (spawned,
    so nothing is inherited) and each is the oracle's serial deterministic solve."""
    import multiprocessing as mp
    jobs = [(n, b) for n in names for b in range(len(G.situations(n)))]
    if workers > 1 and len(jobs) > 1:
        with mp.get_context("spawn").Pool(min(workers, len(jobs))) as pool:
            res = pool.map(_solve_one, jobs, chunksize=1)
    else:
        res = [_solve_one(j) for j in jobs]
    out = {n: ([], [], []) for n in names}
    for (n, _), (f, st, tr) in zip(jobs, res):
        out[n][0].append(f)
        out[n][1].append(st)
        out[n][2].append(tr)
    return out


def main(names):
    sha = {}
    path = os.path.join(HERE, "checksums.json")
    if os.path.exists(path):
        sha = G.load_sha()
    results = run_cases(names, int(os.environ.get("GOLDEN_WORKERS", os.cpu_count() or 1)))
    for name in names:
        fs, stats, traces = results[name]
        if G.storage(name) == "npz":
            arrs = {}
            for b, f in enumerate(fs):
                for fld in G.FIELDS:
                    a = getattr(f, fld)
                    if a is not None:
                        arrs[f"{fld}_{b}"] = a
                arrs[f"trace_{b}"] = traces[b]
            arrs["stats"] = np.array(json.dumps([G.stats_subset(s) for s in stats]))
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrs)
        else:
            sha[name] = G.outputs_sha(fs, stats, traces)
        print(name, [s["iterations"] for s in stats], flush=True)
    with open(path, "w") as fh:
        json.dump(sha, fh, indent=1, sort_keys=True)
    man = {"oracle_sources": {f: sha_file(os.path.join(ROOT, "oracle", f))
                              for f in ("oracle.cpp", "mom_ml.cpp", "mom_ke.cpp", "oracle_common.h")},
           "reference": "GRAL 24.11.2 (GRAL.csproj VersionPrefix), deterministic mode",
           "generator": "tests/golden/make_golden.py"}
    if REFERENCE_TREE and os.path.isdir(REFERENCE_TREE):
        man["reference_sources"] = {f: sha_file(os.path.join(REFERENCE_TREE, f))
                                    for f in REFERENCE_FILES if os.path.exists(os.path.join(REFERENCE_TREE, f))}
    else:
        old = os.path.join(HERE, "MANIFEST.json")
        if os.path.exists(old):
            with open(old) as fh:
                man["reference_sources"] = json.load(fh).get("reference_sources", {})
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as fh:
        json.dump(man, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(G.CASES))
