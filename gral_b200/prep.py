"""Flat-terrain preparation of a prognostic solve (host side, numpy).

Restates what GRAL computes before it calls ``PrognosticFlowfield.Calculate()`` on flat terrain:

* the stretched vertical grid, ``GenerateVerticalGridFlat`` (ProgramFunctions.cs:27-77) with
  ``HOKART[1] = DZK[1]`` (ProgramFunctions.cs:552), in float32 as the reference;
* the surface index KKART from the building heights and KADVMAX (MicroscaleFlat.cs:56-197);
* the prognostic sub-domain mask ADVDOM (ReadGeometryAndDomains.cs:321-347);
* the reference point of the sub-domains (MicroscaleTerrainSearchRefPoint.cs:27-100);
* the initial wind field, zero inside obstacles with the same face rules as
  MicroscaleFlat.cs:83-185.  The vertical profile is a neutral log law scaled to a given speed at
  10 m instead of GRAL's measured-profile power law; both the CUDA solver and the oracle start
  from this same field.

Synthetic inputs only: buildings, inflow and stability are seeded, there is no file IO.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .abi import FieldArrays, StaticArrays

F32 = np.float32


def vertical_grid_flat(dz1: float, stretch: float, top: float = 800.0,
                       max_bound: int = 2048) -> Tuple[int, np.ndarray, np.ndarray]:
    """DZK, HOKART of the flat-terrain grid; returns (NKK, dzk[NKK+2], hokart[NKK+2])."""
    dzk = np.zeros(max_bound, dtype=F32)
    hok = np.zeros(max_bound, dtype=F32)
    dzk[1] = F32(dz1)
    hok[1] = dzk[1]
    s = F32(stretch)
    nkk = 0
    for i in range(2, max_bound):
        dzk[i] = F32(dzk[i - 1] * s)
        hok[i] = F32(hok[i - 1] + dzk[i])
        if hok[i] >= top:
            nkk = i
            break
    nkk = min(nkk, max_bound - 2)
    return nkk, dzk[: nkk + 2].copy(), hok[: nkk + 2].copy()


@dataclass
class Building:
    i0: int   # first 1-based cell index in x
    i1: int   # last cell index in x (inclusive)
    j0: int
    j1: int
    height: float


@dataclass
class Situation:
    """One weather situation: inflow direction/speed/roughness and stability."""
    direction_deg: float = 270.0   # meteorological: wind blowing FROM this direction
    speed_10m: float = 3.0
    z0: float = 0.2
    ustar: float = 0.3
    obukhov: float = 1000.0        # > 0 stable/neutral, < 0 unstable
    potdtdz: float = 0.0


def weather_situations(n: int = 144, seed: int = 3) -> List[Situation]:
    """The batched weather-situation set on a production grid: 36 directions (0-350 deg in 10-deg
    steps) x 4 speeds (0.5/1/2/4 m/s at 10 m), direction outer, z0 0.5 m, u* = 0.1*speed + 0.1,
    stability class drawn per situation from {stable, neutral, unstable} with a seeded generator
    (Obukhov length 50 / 1000 / -50 m, potential temperature gradient 0.01 / 0 / -0.01 K/m); the
    first n of them."""
    rng = np.random.default_rng(seed)
    out = []
    for d in range(36):
        for sp in (0.5, 1.0, 2.0, 4.0):
            cls = int(rng.integers(0, 3))
            out.append(Situation(direction_deg=10.0 * d, speed_10m=sp, z0=0.5, ustar=0.1 * sp + 0.1,
                                 obukhov={0: 50.0, 1: 1000.0, 2: -50.0}[cls],
                                 potdtdz={0: 0.01, 1: 0.0, 2: -0.01}[cls]))
    return out[:n]


@dataclass
class Domain:
    """Everything a solve needs except the per-situation fields."""
    nii: int
    njj: int
    nkk: int
    dxk: float
    dyk: float
    vert_cells_ff: int
    kadvmax: int
    ref: Tuple[int, int]
    static: StaticArrays
    buildings: List[Building] = field(default_factory=list)

    @property
    def cols(self) -> int:
        return (self.nii + 2) * (self.njj + 2)

    def params(self, situation: Optional[Situation] = None, *, model: int = 1, iterations: int = 100,
               iter_min: Optional[int] = None, simd_width: int = 8, quantise: int = 1,
               conv_cadence: int = 100, conv_threshold: float = 0.012, latitude: float = 47.0,
               relax: float = 0.1, relaxp: float = 1.0, building_z0: float = 0.001,
               post_diagnostic: int = 0) -> dict:
        sit = situation or Situation()
        cor = float(F32(2 * 7.29 * 0.00001 * math.sin(abs(latitude) * 3.1415 / 180)))
        return dict(
            nii=self.nii, njj=self.njj, nkk=self.nkk, kadvmax=self.kadvmax,
            vert_cells_ff=self.vert_cells_ff, dxk=self.dxk, dyk=self.dyk,
            turbulence_model=model, simd_width=simd_width,
            iteration_steps_min=iterations if iter_min is None else iter_min,
            iteration_steps_max=iterations, conv_cadence=conv_cadence,
            conv_threshold=conv_threshold, relax=relax, relaxp=relaxp,
            building_z0=building_z0, coriolis=cor, potdtdz=sit.potdtdz,
            ref_i=self.ref[0], ref_j=self.ref[1], quantise=quantise, turb_init=0,
            std_dev_v=1.0, std_dev_w=1.0, bd_lay_height=1000.0, v0_1=float(F32(2.0 * sit.ustar)),
            post_diagnostic=post_diagnostic)


def rasterise(nii: int, njj: int, buildings: List[Building]) -> np.ndarray:
    cutk = np.zeros((nii + 2, njj + 2), dtype=F32)
    for b in buildings:
        cutk[b.i0:b.i1 + 1, b.j0:b.j1 + 1] = np.maximum(cutk[b.i0:b.i1 + 1, b.j0:b.j1 + 1], F32(b.height))
    return cutk


def kkart_from_cutk(cutk: np.ndarray, dzk: np.ndarray, hokart: np.ndarray, nkk: int) -> np.ndarray:
    """KKART = highest k whose cell centre HOKART[k-1] + DZK[k]/2 lies at or below CUTK
    (MicroscaleFlat.cs:86-87, 168-176)."""
    vertk = (hokart[0:nkk] + dzk[1:nkk + 1] * F32(0.5)).astype(F32)   # index k-1 -> level k
    below = vertk[None, None, :] <= cutk[:, :, None]
    kk = np.where(below.any(axis=2), nkk - np.argmax(below[:, :, ::-1], axis=2), 0)
    return kk.astype(np.int16)


def advdom_from_cutk(cutk: np.ndarray, nii: int, njj: int, dxk: float, dyk: float,
                     factor: int = 15) -> np.ndarray:
    """Prognostic sub-domains around every building cell (ReadGeometryAndDomains.cs:321-347)."""
    adv = np.zeros_like(cutk, dtype=np.uint8)
    ii, jj = np.nonzero(cutk[1:nii + 1, 1:njj + 1] > 0)
    for i, j in zip(ii + 1, jj + 1):
        h = cutk[i, j]
        ip = int(F32(factor) * h / F32(dxk))
        jp = int(F32(factor) * h / F32(dyk))
        adv[max(1, i - ip):min(nii, i + ip) + 1, max(1, j - jp):min(njj, j + jp) + 1] = 1
    return adv


def search_reference_point(adv: np.ndarray) -> Tuple[int, int]:
    """Spiral search from the border inwards (MicroscaleTerrainSearchRefPoint.cs:27-100)."""
    xmax, ymax = adv.shape
    searchmax = min(xmax, ymax) // 2
    delta = 1
    i = j = 1
    found = False
    while not found and delta < searchmax:
        i = j = delta
        while j < ymax - delta and not found:
            if adv[i, j] == 1:
                found = True
            else:
                j += 1
        while i < xmax - delta and not found:
            if adv[i, j] == 1:
                found = True
            else:
                i += 1
        while j > delta and not found:
            if adv[i, j] == 1:
                found = True
            else:
                j -= 1
        while i > delta and not found:
            if adv[i, j] == 1:
                found = True
            else:
                i -= 1
        delta += 1
    if not found:
        return (1, 1)
    return (i, j)


def make_domain(nii: int, njj: int, dxk: float, dz1: float, stretch: float, vert_cells_ff: int,
                buildings: List[Building], *, dyk: Optional[float] = None, z0: float = 0.2,
                ustar: float = 0.3, obukhov: float = 1000.0, subdomain_factor: int = 15,
                veg: Optional[np.ndarray] = None, cov: Optional[np.ndarray] = None,
                top: float = 800.0, surface: Optional[np.ndarray] = None) -> Domain:
    dyk = dxk if dyk is None else dyk
    nkk, dzk, hok = vertical_grid_flat(dz1, stretch, top=top)
    cutk = rasterise(nii, njj, buildings)
    if surface is not None:   # blocked cells below a terrain surface, buildings standing on it
        cutk = (cutk + surface.astype(F32)).astype(F32)
    kkart = kkart_from_cutk(cutk, dzk, hok, nkk)
    kmax_b = int(kkart[cutk > 0].max()) if (cutk > 0).any() else 1
    kadvmax = min(nkk, max(1, kmax_b) + vert_cells_ff)
    adv = advdom_from_cutk(cutk, nii, njj, dxk, dyk, subdomain_factor)
    shape2 = (nii + 2, njj + 2)
    st = StaticArrays(
        kkart=kkart, advdom=adv, cutk=cutk,
        cov=np.zeros(shape2, F32) if cov is None else cov.astype(F32),
        z0=np.full(shape2, F32(z0)), z0_init=np.full(shape2, F32(z0)),
        ob_init=np.full(shape2, F32(obukhov)), ust_init=np.full(shape2, F32(ustar)),
        dzk=dzk, hokart=hok)
    if veg is not None:
        st.veg = np.ascontiguousarray(veg, dtype=F32)
        st.veg_mask = (st.veg.max(axis=2) > 0).astype(np.uint8)
    ref = search_reference_point(adv)
    return Domain(nii, njj, nkk, dxk, dyk, vert_cells_ff, kadvmax, ref, st, buildings)


def log_profile(z: np.ndarray, speed_10m: float, z0: float) -> np.ndarray:
    return speed_10m * np.maximum(np.log(np.maximum(z, 1e-6) / z0), 0.0) / math.log(10.0 / z0)


def _masked_fields(dom: Domain, u: np.ndarray, v: np.ndarray, dtype):
    """UK, VK of the domain from per-level profiles u, v (index = level), with the obstacle rules
    of MicroscaleFlat.cs: zero inside obstacles and on faces shared with an obstacle cell, the
    east/north edge copies, zero at level 0."""
    nii, njj, nkk = dom.nii, dom.njj, dom.nkk
    st = dom.static
    shape = (nii + 2, njj + 2, nkk + 2)
    uk = np.zeros(shape, dtype)
    vk = np.zeros(shape, dtype)
    vertk = np.zeros(nkk + 2, F32)
    vertk[1:nkk + 1] = st.hokart[0:nkk] + st.dzk[1:nkk + 1] * F32(0.5)
    cut = st.cutk
    inside = vertk[None, None, :] <= cut[:, :, None]             # cell (i,j,k) inside an obstacle
    inside[..., 0] = False
    inside[..., nkk + 1] = False
    uk[1:nii + 1, 1:njj + 1, :] = u
    vk[1:nii + 1, 1:njj + 1, :] = v
    uk[inside] = 0
    vk[inside] = 0
    uk[2:nii + 1][inside[1:nii]] = 0                              # west neighbour is an obstacle
    vk[:, 2:njj + 1][inside[:, 1:njj]] = 0                        # south neighbour is an obstacle
    uk[nii + 1, 1:njj + 1, :] = uk[nii, 1:njj + 1, :]
    vk[1:nii + 1, njj + 1, :] = vk[1:nii + 1, njj, :]
    uk[..., 0] = 0
    vk[..., 0] = 0
    return uk, vk


def _cell_heights(dom: Domain) -> np.ndarray:
    nkk = dom.nkk
    vertk = np.zeros(nkk + 2, F32)
    vertk[1:nkk + 1] = dom.static.hokart[0:nkk] + dom.static.dzk[1:nkk + 1] * F32(0.5)
    return vertk


def initial_fields(dom: Domain, sit: Situation, model: int = 1) -> FieldArrays:
    """Initial UK/VK/WK (and TURB/TDISS buffers) with the obstacle rules of MicroscaleFlat.cs."""
    nii, njj, nkk = dom.nii, dom.njj, dom.nkk
    shape = (nii + 2, njj + 2, nkk + 2)
    vertk = _cell_heights(dom)
    sp = log_profile(vertk.astype(np.float64), sit.speed_10m, sit.z0)
    th = math.radians(sit.direction_deg)
    u = (-sp * math.sin(th)).astype(F32)
    v = (-sp * math.cos(th)).astype(F32)
    u[0] = v[0] = 0
    u[nkk + 1] = v[nkk + 1] = 0
    uk, vk = _masked_fields(dom, u, v, F32)
    wk = np.zeros(shape, F32)
    turb = tdiss = None
    if model != 1:
        turb = np.zeros(shape, F32)
        tdiss = np.zeros(shape, F32)
    return FieldArrays(uk, vk, wk, turb, tdiss)


KARMAN = 0.4


def inflow_tangents(dom: Domain, sit: Situation) -> dict:
    """Derivatives of the initial UK, VK of ``initial_fields`` with respect to the inflow
    parameters of the neutral log-law profile u(z) = (u*/0.4) ln(z/z0) along the direction
    (u* = 0.4 * speed_10m / ln(10/z0)): name -> (dUK, dVK) in float64 for "ustar" (z0 and the
    direction fixed), "z0" (u* and the direction fixed) and "direction_deg" (per degree)."""
    nkk = dom.nkk
    z = _cell_heights(dom).astype(np.float64)
    ustar = KARMAN * sit.speed_10m / math.log(10.0 / sit.z0)
    lnz = np.log(np.maximum(z, 1e-6) / sit.z0)
    pos = lnz > 0
    sp = np.where(pos, ustar / KARMAN * lnz, 0.0)
    th = math.radians(sit.direction_deg)
    dsp = {"ustar": np.where(pos, lnz / KARMAN, 0.0), "z0": np.where(pos, -ustar / (KARMAN * sit.z0), 0.0)}
    out = {}
    for name, d in dsp.items():
        du, dv = -d * math.sin(th), -d * math.cos(th)
        du[0] = dv[0] = du[nkk + 1] = dv[nkk + 1] = 0.0
        out[name] = _masked_fields(dom, du, dv, np.float64)
    du, dv = -sp * math.cos(th) * math.pi / 180.0, sp * math.sin(th) * math.pi / 180.0
    du[0] = dv[0] = du[nkk + 1] = dv[nkk + 1] = 0.0
    out["direction_deg"] = _masked_fields(dom, du, dv, np.float64)
    return out


def inflow_gradient(dom: Domain, sit: Situation, dj_duk0: np.ndarray, dj_dvk0: np.ndarray) -> dict:
    """dJ/d(u*, z0, direction) from the cotangents of the initial UK, VK (chain rule through
    ``inflow_tangents``)."""
    return {name: float((du * dj_duk0).sum() + (dv * dj_dvk0).sum())
            for name, (du, dv) in inflow_tangents(dom, sit).items()}


# --------------------------------------------------------------------------------------------
# Named workloads
# --------------------------------------------------------------------------------------------

def cube_domain(n: int = 100, dx: float = 2.0, dz1: float = 2.0, stretch: float = 1.01,
                vert_cells_ff: int = 20, size_m: float = 20.0, height: float = 20.0,
                **kw) -> Domain:
    """One cube building at the domain centre (100x100x20 at 2 m, 20 m cube by default)."""
    nb = int(round(size_m / dx))
    c0 = n // 2 - nb // 2 + 1
    b = Building(c0, c0 + nb - 1, c0, c0 + nb - 1, height)
    return make_domain(n, n, dx, dz1, stretch, vert_cells_ff, [b], **kw)


def random_buildings(nii: int, njj: int, dx: float, count: int, seed: int,
                     foot_m: Tuple[float, float] = (10.0, 40.0),
                     height_m: Tuple[float, float] = (10.0, 30.0), margin_cells: int = 6,
                     gap_cells: int = 2) -> List[Building]:
    """Non-overlapping rectangles by rejection sampling (seeded numpy PCG64)."""
    rng = np.random.default_rng(seed)
    occ = np.zeros((nii + 2, njj + 2), dtype=bool)
    out: List[Building] = []
    tries = 0
    while len(out) < count and tries < 200000:
        tries += 1
        wx = int(round(rng.uniform(*foot_m) / dx))
        wy = int(round(rng.uniform(*foot_m) / dx))
        wx, wy = max(wx, 1), max(wy, 1)
        i0 = int(rng.integers(1 + margin_cells, nii - margin_cells - wx + 1))
        j0 = int(rng.integers(1 + margin_cells, njj - margin_cells - wy + 1))
        a0, a1 = max(1, i0 - gap_cells), min(nii, i0 + wx - 1 + gap_cells)
        b0, b1 = max(1, j0 - gap_cells), min(njj, j0 + wy - 1 + gap_cells)
        if occ[a0:a1 + 1, b0:b1 + 1].any():
            continue
        occ[i0:i0 + wx, j0:j0 + wy] = True
        h = float(F32(rng.uniform(*height_m)))
        out.append(Building(i0, i0 + wx - 1, j0, j0 + wy - 1, h))
    return out


def city_domain(n: int = 400, dx: float = 2.0, dz1: float = 2.0, stretch: float = 1.05,
                vert_cells_ff: int = 30, n_buildings: int = 64, seed: int = 2, **kw) -> Domain:
    """Production-size grid: 400x400 cells at 2 m, 64 seeded buildings, 10-30 m tall."""
    bl = random_buildings(n, n, dx, n_buildings, seed)
    return make_domain(n, n, dx, dz1, stretch, vert_cells_ff, bl, **kw)


def adjoint_domain(n: int = 200, dx: float = 2.0, dz1: float = 2.0, stretch: float = 1.05, vert_cells_ff: int = 25,
                   n_buildings: int = 30, veg_fraction: float = 0.2, veg_max: float = 0.5, seed: int = 5) -> Domain:
    """The differentiation workload: an n x n grid at 2 m (first layer 2 m, stretching 1.05),
    seeded buildings, and a vegetation drag density over `veg_fraction` of the columns: a smooth
    random field in [0, veg_max] m^-1 (sums of Gaussian bumps, thresholded to the wanted cover) on
    the levels of a 2-15 m canopy, with cover 0.5 where it is set."""
    rng = np.random.default_rng(7000 + seed)
    fmax = min(40.0, (n - 2 * 6 - 2) * dx / 2)        # footprints 10-40 m, narrowed on small grids
    bl = random_buildings(n, n, dx, n_buildings, seed, foot_m=(min(10.0, fmax), fmax),
                          height_m=(10.0, 30.0) if n >= 100 else (4.0, 14.0))
    nkk, dzk, hok = vertical_grid_flat(dz1, stretch)
    xs = np.arange(n + 2, dtype=np.float64)
    field2 = np.zeros((n + 2, n + 2))
    for _ in range(max(4, n // 8)):
        cx, cy, sg = rng.uniform(0, n), rng.uniform(0, n), rng.uniform(2.0, max(3.0, n / 10))
        field2 += rng.uniform(0.3, 1.0) * np.exp(-((xs[:, None] - cx) ** 2 + (xs[None, :] - cy) ** 2) / (2 * sg * sg))
    field2[0, :] = field2[:, 0] = field2[n + 1, :] = field2[:, n + 1] = 0
    inner = field2[1:n + 1, 1:n + 1]
    thr = np.quantile(inner, 1.0 - veg_fraction)
    dens = np.where(field2 > thr, (field2 - thr) / max(float(inner.max() - thr), 1e-12), 0.0) * veg_max
    veg = np.zeros((n + 2, n + 2, nkk + 2), F32)
    zc = hok[0:nkk + 1] + 0.5 * dzk[1:nkk + 2]
    canopy = (zc >= 0.0) & (zc <= 15.0)
    for k in range(1, nkk + 1):
        if canopy[k - 1]:
            veg[:, :, k - 1] = dens.astype(F32)
    cov = np.where(dens > 0, F32(0.5), F32(0)).astype(F32)
    return make_domain(n, n, dx, dz1, stretch, vert_cells_ff, bl, veg=veg, cov=cov)


def probe_misfit(dom: Domain, fields, n_probes: int = 1000, seed: int = 11, noise: float = 0.1):
    """Seeded probe cells (i, j, k) inside the prognostic sub-domains, above the surface and within
    the prognostic levels, and targets u_target = the given fields there plus seeded noise, for the
    misfit J = sum over probes of |(U, V, W) - target|^2.  Returns (flat indices, targets [n, 3])."""
    rng = np.random.default_rng(seed)
    st = dom.static
    cand = []
    for i in range(3, dom.nii - 1):
        for j in range(3, dom.njj - 1):
            if st.advdom[i, j] == 1:
                cand.append((i, j))
    idx = []
    nk2 = dom.nkk + 2
    for q in rng.integers(0, len(cand), n_probes):
        i, j = cand[int(q)]
        kk = int(st.kkart[i, j])
        k = int(rng.integers(kk + 2, kk + dom.vert_cells_ff))
        idx.append((i * (dom.njj + 2) + j) * nk2 + k)
    idx = np.array(idx, np.int64)
    tgt = np.stack([a.reshape(-1)[idx] for a in (fields.uk, fields.vk, fields.wk)], axis=1).astype(np.float64)
    tgt = tgt + rng.normal(0.0, noise, tgt.shape)
    return idx, tgt


def misfit_and_cotangent(idx: np.ndarray, tgt: np.ndarray, uk, vk, wk, dtype=np.float64):
    """J = sum |(U, V, W)(probe) - target|^2 and its cotangents dJ/dUK, dJ/dVK, dJ/dWK."""
    J = 0.0
    gs = []
    for q, a in enumerate((uk, vk, wk)):
        r = a.reshape(-1)[idx].astype(np.float64) - tgt[:, q]
        J += float((r * r).sum())
        g = np.zeros(a.size, np.float64)
        np.add.at(g, idx, 2.0 * r)
        gs.append(g.reshape(a.shape).astype(dtype))
    return J, gs


def hilly_domain(nii: int, njj: int, dx: float, vert_cells_ff: int, seed: int, n_hills: Optional[int] = None,
                 n_buildings: Optional[int] = None, dz1: float = 2.0, stretch: float = 1.05) -> Domain:
    """Instance of the uneven-domain set: 1-5 Gaussian hills (5-50 m high, sigma 30-150 m) and
    0-80 buildings (counts seeded unless given), the hill surface blocked like buildings (CUTK =
    surface + building height) so that the flat-terrain solver sees the terrain through KKART."""
    rng = np.random.default_rng(5000 + seed)
    nh = int(rng.integers(1, 6)) if n_hills is None else n_hills
    nb = int(rng.integers(0, 81)) if n_buildings is None else n_buildings
    xs = (np.arange(nii + 2, dtype=np.float64) - 0.5) * dx
    ys = (np.arange(njj + 2, dtype=np.float64) - 0.5) * dx
    surf = np.zeros((nii + 2, njj + 2))
    for _ in range(nh):
        h, sg = rng.uniform(5.0, 50.0), rng.uniform(30.0, 150.0)
        cx, cy = rng.uniform(0, nii * dx), rng.uniform(0, njj * dx)
        surf += h * np.exp(-((xs[:, None] - cx) ** 2 + (ys[None, :] - cy) ** 2) / (2 * sg * sg))
    surf[0, :] = surf[:, 0] = 0
    surf[nii + 1, :] = surf[:, njj + 1] = 0
    # footprints 10-40 m, narrowed to what fits the grid between its margins
    fmax = min(40.0, (min(nii, njj) - 2 * 3 - 2) * dx / 2)
    bl = random_buildings(nii, njj, dx, nb, seed, foot_m=(min(10.0, fmax), fmax), margin_cells=3,
                          gap_cells=1) if nb and fmax >= dx else []
    top = max(800.0, float(surf.max()) + 400.0)
    return make_domain(nii, njj, dx, dz1, stretch, vert_cells_ff, bl, surface=surf.astype(F32), top=top)


def random_situation(seed: int) -> "Situation":
    """Random inflow direction, 10 m speed and roughness (z0 0.05-1 m), neutral."""
    rng = np.random.default_rng(7000 + seed)
    return Situation(direction_deg=float(rng.uniform(0, 360)), speed_10m=float(rng.uniform(0.5, 4.0)),
                     z0=float(rng.uniform(0.05, 1.0)))


def small_domain(nii: int = 16, njj: int = 14, seed: int = 0, n_buildings: int = 3,
                 vert_cells_ff: int = 12, stretch: float = 1.05, dx: float = 2.0,
                 with_veg: bool = False, **kw) -> Domain:
    """Small seeded test grid with a few buildings of mixed heights (and optional vegetation)."""
    rng = np.random.default_rng(1000 + seed)
    bl = random_buildings(nii, njj, dx, n_buildings, seed, foot_m=(4.0, 8.0), height_m=(3.0, 16.0),
                          margin_cells=3, gap_cells=1)
    veg = cov = None
    if with_veg:
        nkk, _, _ = vertical_grid_flat(2.0, stretch)
        veg = np.zeros((nii + 2, njj + 2, nkk + 2), F32)
        cov = np.zeros((nii + 2, njj + 2), F32)
        for _ in range(3):
            i = int(rng.integers(3, nii - 2)); j = int(rng.integers(3, njj - 2))
            veg[i - 1:i + 2, j - 1:j + 2, 1:6] = F32(rng.uniform(0.05, 0.5))
            cov[i - 1:i + 2, j - 1:j + 2] = F32(rng.uniform(0.2, 0.9))
    return make_domain(nii, njj, dx, 2.0, stretch, vert_cells_ff, bl, veg=veg, cov=cov, **kw)
