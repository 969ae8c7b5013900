"""The discrete adjoint's CPU side: the hand-derived per-level derivatives of the library's
model-1 momentum rows, the FP64 twin of the oracle, its tape-based gradient, and the inflow
tangents of the initial field.

* ``tests/native/adj_level_check.cpp`` compiles the library's level functions
  (``gral_b200/csrc/adj_level.cuh``) for the host and checks every vector-Jacobian product against
  central differences of the forward row in double precision.
* The FP64 twin (``oracle_twin_forward``) runs the oracle's own model-1 operations in double: it
  must agree with the float oracle (no rounding) to float precision.
* Its reverse-mode gradient (tape differentiation of the same operations) must agree with FP64
  central differences of the twin along random directions of VEG and the initial fields.
* ``prep.inflow_tangents`` must agree with differences of the initial-field builder.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from gral_b200 import prep
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_level_vjps_match_central_differences():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "adj_level_check")
        subprocess.run([gxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "gral_b200", "csrc"), "-o", exe,
                        os.path.join(ROOT, "tests", "native", "adj_level_check.cpp")], check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("0 mismatches") == 3, r.stdout


def small_case(iterations=6, seed=3):
    dom = prep.small_domain(16, 16, seed=seed, with_veg=True)
    sit = prep.Situation(direction_deg=200.0, speed_10m=3.0)
    f = prep.initial_fields(dom, sit)
    p = dom.params(sit, model=1, iterations=iterations, quantise=0)
    return dom, sit, f, p


def test_twin_agrees_with_the_float_oracle():
    dom, sit, f, p = small_case()
    fo = f.copy()
    O.solve(p, dom.static, fo)
    x0 = (f.uk.astype(np.float64), f.vk.astype(np.float64), f.wk.astype(np.float64))
    u, v, w = O.twin_forward(p, dom.static, f, x0, dom.static.veg.astype(np.float64), p["iteration_steps_max"])
    for a, b in ((u, fo.uk), (v, fo.vk), (w, fo.wk)):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


def test_twin_gradient_matches_central_differences():
    dom, sit, f, p = small_case(iterations=6)
    n = p["iteration_steps_max"]
    x0 = (f.uk.astype(np.float64), f.vk.astype(np.float64), f.wk.astype(np.float64))
    veg = dom.static.veg.astype(np.float64)
    u, v, w = O.twin_forward(p, dom.static, f, x0, veg, n)
    idx, tgt = prep.probe_misfit(dom, prep.FieldArrays(u, v, w), n_probes=60, seed=2)

    def J(xx, vg):
        return prep.misfit_and_cotangent(idx, tgt, *O.twin_forward(p, dom.static, f, xx, vg, n))[0]

    _, g = prep.misfit_and_cotangent(idx, tgt, u, v, w)
    d_uk0, d_vk0, d_wk0, d_veg = O.twin_vjp(p, dom.static, f, x0, veg, n, g)
    rng = np.random.default_rng(0)
    mask = (veg > 0).astype(np.float64)
    worst = 0.0
    for _ in range(4):
        dv = rng.normal(size=veg.shape) * mask * 0.05
        du = rng.normal(size=u.shape) * 0.01 * (np.abs(x0[0]) > 0)
        h = 1e-4
        fd = (J((x0[0] + h * du, x0[1], x0[2]), veg + h * dv) - J((x0[0] - h * du, x0[1], x0[2]), veg - h * dv)) / (2 * h)
        ad = float((d_veg * dv).sum() + (d_uk0 * du).sum())
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-12))
    assert worst <= 1e-3, worst


def test_inflow_tangents_match_differences():
    dom = prep.small_domain(16, 14, seed=1)
    sit = prep.Situation(direction_deg=250.0, speed_10m=3.0, z0=0.2)
    z = prep._cell_heights(dom).astype(np.float64)

    def fields(ustar, z0, deg):
        sp = ustar / prep.KARMAN * np.maximum(np.log(np.maximum(z, 1e-6) / z0), 0.0)
        th = np.radians(deg)
        u, v = -sp * np.sin(th), -sp * np.cos(th)
        u[0] = v[0] = u[-1] = v[-1] = 0.0
        return prep._masked_fields(dom, u, v, np.float64)

    us = prep.KARMAN * sit.speed_10m / np.log(10.0 / sit.z0)
    t = prep.inflow_tangents(dom, sit)
    h = 1e-6
    for name, args in (("ustar", (0, h)), ("z0", (1, h)), ("direction_deg", (2, 1e-4))):
        q, e = args
        base = [us, sit.z0, sit.direction_deg]
        hi, lo = list(base), list(base)
        hi[q] += e
        lo[q] -= e
        fu, fv = fields(*hi)
        gu, gv = fields(*lo)
        du, dv = t[name]
        np.testing.assert_allclose(du, (fu - gu) / (2 * e), rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(dv, (fv - gv) / (2 * e), rtol=1e-5, atol=1e-7)
