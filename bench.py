"""Benchmark of the B200 prognostic microscale flow solver.

Metric: Mcell-iterations/s (nominal cells = ADVDOM columns x VertCellsFF, per SIMPLE iteration).
A "step" is one SIMPLE iteration over the whole workload.  Default workload: the production-size
plain solve, 400x400 cells at 2 m with 30 prognostic levels (stretch 1.05, NKK 63, KADVMAX 41),
64 seeded buildings 10-30 m tall, inflow from 225 deg at 2 m/s (z0 0.5 m, neutral), mixing-length
model; synthetic, seeded inputs.

  value      device-resident throughput: K timed iterations after W warm-up iterations, CUDA
             events on the solver's stream, inputs already in HBM (working set > L2).
  e2e        one full solve through the public C ABI (gral_prog_solve: pinned host buffers in,
             set-up, 500 SIMPLE iterations, post-checks, fields back to the host), host-timed.
  roofline   dominant kernel's algorithmic bytes per launch / its mean CUDA-event duration,
             against the measured HBM copy bandwidth.
  batched    the batched form on the same grid: the 144-situation weather set (36 directions x 4
             speeds, seeded stability) as one batch, 10 device-timed iterations (throughput, phase
             split, roofline), and `to_stop`: the whole set solved to its stop rule (_delta < 1e-3
             tested every 100 iterations, or 800 iterations) in one batched call against plain
             single-situation calls, both host-timed end to end, in situations/hour.
  cpu_baseline  the C++ restatement on all host cores, in the faster of its two host forms (one
             situation over all threads in the reference's racy work split, or one single-threaded
             situation per core), on a bounded sample of the same workload.
  prep       the flow-field set-up before the solve (sub-domains, flat-terrain initial field,
             vegetation) on the same grid: device kernel time (CUDA events) against HBM bandwidth,
             host-timed calls including the copies, and the oracle restatement on one core.
  wind       the wind at 2^20 random particle positions interpolated from the solved field
             (IntWindCalculate): device kernel time, the call with the host copies, the oracle on
             one core.
  instances  independent situations on grids of different sizes (the uneven-domain batch: grids
             log-uniform 128x128x20 .. 512x512x40 at 2-4 m, hills and buildings, random inflow),
             solved one at a time and side by side (gral_prog_solve_instances), host-timed.
  adjoint    the discrete adjoint (gral_prog_vjp) of 200 unrolled iterations on a 200x200x25 grid
             with vegetation drag over 20 % of the columns and a 1000-probe misfit: device times of
             the forward with checkpoints and of the vector-Jacobian product, and their ratio.
  gff        the flow-field cache writer/reader (GFFWrite.cs / GFFRead.cs formats) on the same
             grid: device pack kernel per format (CUDA events, L2 flushed before each launch)
             against HBM bandwidth, the host-timed pack into pinned memory and read back, and
             the numpy restatement of the writer timed on one core.

`--impl reference` times the CPU path on this host's cores and prints the same metric: the C#
reference cannot run here (no .NET SDK), so its C++ restatement (-O3 -march=native, built on the
host) runs each step both as one situation with its sweeps over all host threads in the
reference's default (racy) work split and as one single-threaded situation per core in separate
processes; the faster form is the value.
Multi-GPU (torchrun): every rank solves its own replica of the workload (a single situation does
not shard); value = all ranks' cell-iterations / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-iterations/s on 1 B200 (batched vs plain, ≤1e-4 rel err); HBM fraction"
UNIT = "Mcell-iterations/s"
BYTES_PER_CELL = {"pressure": 24, "velcorr": 28, "u": 20, "v": 20, "w": 20,   # model 1
                  "pvau": 24 + 28 + 20}   # fused pressure + velocity correction + averages + U


def workload(name: str, grid: int = 400):
    from gral_b200 import prep
    if name == "production" and grid != 400:
        dom = prep.city_domain(n=grid, dx=2.0, dz1=2.0, stretch=1.05, vert_cells_ff=30,
                               n_buildings=max(1, 64 * grid * grid // 160000), seed=2)
        sit = prep.Situation(direction_deg=225.0, speed_10m=2.0, z0=0.5, ustar=0.3)
        return dom, sit, 500, f"{grid}x{grid}x30 at 2 m, stretch 1.05, seeded buildings, 225 deg 2 m/s, 500 iterations"
    if name == "batched" and grid != 400:
        dom = prep.city_domain(n=grid, dx=2.0, dz1=2.0, stretch=1.05, vert_cells_ff=30,
                               n_buildings=max(1, 64 * grid * grid // 160000), seed=2)
        return dom, None, 800, f"batched situations on a {grid}x{grid}x30 grid"
    if name == "production":
        dom = prep.city_domain(n=400, dx=2.0, dz1=2.0, stretch=1.05, vert_cells_ff=30, n_buildings=64, seed=2)
        sit = prep.Situation(direction_deg=225.0, speed_10m=2.0, z0=0.5, ustar=0.3)
        return dom, sit, 500, "400x400x30 at 2 m, stretch 1.05, 64 buildings, 225 deg 2 m/s, z0 0.5, 500 iterations"
    if name == "batched":
        dom = prep.city_domain(n=400, dx=2.0, dz1=2.0, stretch=1.05, vert_cells_ff=30, n_buildings=64, seed=2)
        return dom, None, 800, ("144 situations (36 directions x 4 speeds, seeded stability) on the 400x400x30 "
                                "production grid, up to 800 iterations")
    if name == "cube":
        dom = prep.cube_domain(n=100, dx=2.0, dz1=2.0, stretch=1.01, vert_cells_ff=20, z0=0.2, ustar=0.3)
        sit = prep.Situation(direction_deg=270.0, speed_10m=3.0, z0=0.2, ustar=0.3)
        return dom, sit, 100, "100x100x20 at 2 m, stretch 1.01, one 20 m cube, 270 deg 3 m/s, z0 0.2, 100 iterations"
    raise SystemExit(f"unknown workload {name}")


def batched_situations(n: int = 144, seed: int = 3):
    """36 directions (0-350 deg in 10-deg steps) x 4 speeds (0.5/1/2/4 m/s at 10 m), stability
    classes drawn from {stable, neutral, unstable} with a seeded generator; first n of them."""
    from gral_b200 import prep
    return prep.weather_situations(n, seed)


def rank_situations(base_situation, batch: int, rank: int, world: int):
    """Situations one rank solves.  A single situation does not shard: every rank solves its own
    replica.  Batches shard by situation with no exchange during the solve (weak scaling): rank 0
    solves the 144-situation set itself, rank r the same 36 x 4 grid of directions and speeds turned
    by r * 10/world degrees, so every rank's situations are distinct and the per-rank work fixed."""
    from gral_b200 import prep
    if base_situation is not None:
        return [base_situation]
    out = []
    for x in batched_situations(batch):
        d = (x.direction_deg + rank * 10.0 / max(world, 1)) % 360.0
        out.append(prep.Situation(direction_deg=d, speed_10m=x.speed_10m, z0=x.z0, ustar=x.ustar,
                                  obukhov=x.obukhov, potdtdz=x.potdtdz))
    return out


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank float over the default process group (identity without one)."""
    import torch
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def nominal_cells(dom) -> int:
    adv = dom.static.advdom[1:dom.nii + 1, 1:dom.njj + 1]
    return int((adv == 1).sum()) * dom.vert_cells_ff


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(layout: str, phase: str, cells: int):
    """DRAM bytes (read + write) per launch of the phase's kernel from the committed ncu summary
    ``profiles/dram_traffic.txt`` (lines: layout phase kernel bytes cells_of_capture), scaled to
    `cells` when the capture ran on a smaller case; None when that kernel was not captured."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as fh:
            for line in fh:
                parts = line.split()
                if len(parts) >= 5 and parts[0] == layout and parts[1] == phase:
                    return round(float(parts[3]) * cells / float(parts[4]))
    except (OSError, ValueError):
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "", 1).isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def pinned_fields(f):
    """Copies of the initial fields in page-locked host memory (torch pinned tensors)."""
    import torch
    from gral_b200.abi import FieldArrays

    def pin(a):
        if a is None:
            return None
        t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
        n = t.numpy()
        n[...] = a
        return n
    return FieldArrays(pin(f.uk), pin(f.vk), pin(f.wk), pin(f.turb), pin(f.tdiss))


def host_cpu() -> dict:
    """The host's CPU model (first `model name` of /proc/cpuinfo) and logical CPU count."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.lower().startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "host_threads": os.cpu_count() or 1}


def cpu_sample(workload_name: str, iterations: int, threaded: bool = True):
    """The CPU restatement on `iterations` SIMPLE iterations of one situation of the workload;
    returns (Mcell-it/s, seconds, threads).  threaded: the racy-order build with the sweeps over all
    host threads (-O3 -march=native, built here), the analogue of the reference's default parallel
    mode; otherwise the deterministic single-threaded oracle."""
    from gral_b200 import prep
    from oracle import oracle as O
    dom, sit, _, _ = workload(workload_name)
    p = dom.params(sit, model=1, iterations=iterations, iter_min=iterations)
    f = prep.initial_fields(dom, sit)
    t0 = time.perf_counter()
    O.solve(p, dom.static, f, threaded=threaded)
    dt = time.perf_counter() - t0
    threads = O.threads_used() if threaded else 1
    return nominal_cells(dom) * iterations / dt / 1e6, dt, threads


CPU_KIND_TEXT = ("C++ restatement of the reference's solver, -O3 -march=native, built on this host; a "
                 "restatement, not the reference (no .NET SDK on the host)")


def _one_thread_env():
    os.environ["ORACLE_THREADS"] = "1"


def _cpu_worker(job):
    name, iters = job
    return cpu_sample(name, iters)


class CpuBaseline:
    """The CPU path on every host core in the two ways a host runs it: one situation with the sweeps
    split over all threads in the reference's default (racy) work split -- what one GRAL process
    does -- and one single-threaded situation per core in independent processes -- what several
    GRAL processes on one host do.  The faster of the two is the baseline."""

    def __init__(self, workload_name: str, iters: int):
        import multiprocessing as mp
        from oracle import oracle as O
        O.build_threaded()
        self.name = workload_name if workload_name != "batched" else "production"
        self.iters = iters
        self.cores = os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.cores, initializer=_one_thread_env)

    def close(self):
        self.pool.close()
        self.pool.join()

    def step(self):
        """One sample of each form: (threaded Mcell-it/s, threads, seconds; processes Mcell-it/s, seconds)."""
        v_t, dt_t, thr = cpu_sample(self.name, self.iters)
        t0 = time.perf_counter()
        res = self.pool.map(_cpu_worker, [(self.name, self.iters)] * self.cores, chunksize=1)
        dt_p = time.perf_counter() - t0
        dom, _, _, _ = workload(self.name)
        v_p = nominal_cells(dom) * self.iters * self.cores / dt_p / 1e6
        return v_t, thr, dt_t, v_p, dt_p

    def describe(self, v_t, thr, dt_t, v_p, dt_p):
        best = "threaded" if v_t >= v_p else "processes"
        return {"value": round(max(v_t, v_p), 4), "unit": UNIT, "cores": self.cores, "kind": "port",
                "form": best,
                "sample": (f"{self.iters} SIMPLE iterations (set-up included) of one situation with its sweeps over "
                           f"{thr} threads in the reference's default work split: {v_t:.3f} Mcell-it/s ({dt_t:.1f} s); "
                           f"{self.cores} situations in {self.cores} single-threaded processes: {v_p:.3f} Mcell-it/s "
                           f"({dt_p:.1f} s); the faster is the baseline; {CPU_KIND_TEXT}"),
                "threaded": round(v_t, 4), "processes": round(v_p, 4), **host_cpu()}


def run_reference(args, rank, world):
    """The reference's CPU path on this host's cores: the C# solver cannot run here (no .NET SDK),
    so its restatement runs each step in both host forms (CpuBaseline), set-up included, for
    args.ref_iters SIMPLE iterations per situation."""
    if rank != 0:
        return
    cb = CpuBaseline(args.workload, args.ref_iters)
    try:
        for _ in range(args.warmup):
            cb.step()
        samples = [cb.step() for _ in range(args.steps)]
    finally:
        cb.close()
    med = [statistics.median(x[q] for x in samples) for q in range(5)]
    desc = cb.describe(med[0], samples[0][1], med[2], med[3], med[4])
    value = desc["value"]
    dom, _, _, wdesc = workload(args.workload)
    cells = nominal_cells(dom)
    per_step = cells * args.ref_iters / (value * 1e6)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": args.workload, "description": wdesc,
                                       "cells_per_situation": cells, "iterations_per_situation": args.ref_iters},
        "cpu_baseline": desc,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def device_run(dom, sits, steps: int, warmup: int, local: int, model: int = 1):
    """Load `sits` on one GPU, run `warmup` untimed then `steps` timed SIMPLE iterations (CUDA
    events on the solver's stream, barrier + synchronize on both sides); returns the max-over-ranks
    time, the phase split and the store statistics."""
    import torch
    import torch.distributed as td
    from gral_b200 import prep
    from gral_b200.prognostic import PrognosticSolver
    dist = td.is_available() and td.is_initialized()
    total = warmup + steps
    # room for the autotuner's trial iterations (one per launch variant) before the timed ones
    ps = [dom.params(x, model=model, iterations=total + 32, iter_min=total + 32) for x in sits]
    fs = [prep.initial_fields(dom, x, model) for x in sits]
    solver = PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=len(sits))
    try:
        solver.load(ps, dom.static, fs)
        solver.iterate_timed(warmup)
        if dist:
            td.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            tot_ms, phases = solver.iterate_timed(steps)
        torch.cuda.synchronize()
        if dist:
            td.barrier()
        st = solver.store(fs)[0]
    finally:
        solver.close()
    return max_over_ranks(tot_ms, "cuda"), tot_ms, phases, st, clk.summary()


def roofline(cells: int, steps: int, phases: dict, layout: str):
    cand = {k: v for k, v in phases.items() if k in BYTES_PER_CELL and v > 0}
    dom_k = max(cand, key=cand.get)
    per_launch_s = cand[dom_k] / steps / 1e3
    alg_bytes = cells * BYTES_PER_CELL[dom_k]
    achieved = alg_bytes / per_launch_s / 1e9
    peak, peak_kind = measured_peak()
    it_ms = sum(phases.values()) / steps
    it_bytes = cells * 112   # pressure 24 + velocity correction 28 + U, V, W 20 each
    return {"bound": "hbm", "kernel": dom_k, "achieved": round(achieved, 2), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 5),
            "traffic": profile_traffic(layout, dom_k, cells), "alg_bytes_per_launch": alg_bytes,
            "hbm_frac_iteration": round(it_bytes / (it_ms / 1e3) / 1e9 / peak, 5)}


def gff_measure(dom, sit, repeats: int = 10):
    """Flow-field cache payloads of one solved situation of `dom` (rank 0 only)."""
    import torch
    from gral_b200 import prep
    from gral_b200.abi import FieldArrays
    from gral_b200.prognostic import GFF_COLUMNS, GFF_LEVELS, GFF_TERRAIN, PrognosticSolver
    from oracle import gff as O

    f = prep.initial_fields(dom, sit)
    peak, peak_kind = measured_peak()
    out = {"workload": f"one situation, {dom.nii}x{dom.njj}x{dom.nkk} grid, fields resident after a store",
           "formats": {}}
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        s.load([dom.params(sit, iterations=1)], dom.static, [f])
        s.store([f])
        for mode, name in ((GFF_COLUMNS, "columns_-1"), (GFF_LEVELS, "levels_-2"), (GFF_TERRAIN, "terrain_-3")):
            nbytes = s.gff_size(mode)
            words = (nbytes - 32) // 2
            kk_words = dom.nii * dom.njj if mode == GFF_TERRAIN else 0
            # per value word: one float read (4 B) and one int16 written (2 B); KKART words 2 B each way
            alg = 6 * (words - kk_words) + 4 * kk_words
            s.gff_pack_timed(0, mode, 3)
            ms = s.gff_pack_timed(0, mode, repeats)
            buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy()
            s.gff_pack(0, mode, 225.0, 2.0, 4, out=buf)
            t0 = time.perf_counter()
            for _ in range(repeats):
                s.gff_pack(0, mode, 225.0, 2.0, 4, out=buf)
            pack_ms = (time.perf_counter() - t0) / repeats * 1e3
            uk, vk, wk = (torch.empty(f.uk.shape, dtype=torch.float32, pin_memory=True).numpy() for _ in range(3))
            tgt = FieldArrays(uk, vk, wk)
            s.gff_unpack(buf, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart, out=tgt)
            t0 = time.perf_counter()
            for _ in range(repeats):
                s.gff_unpack(buf, dom.nii, dom.njj, dom.nkk, dom.dxk, kkart=dom.static.kkart, out=tgt)
            unpack_ms = (time.perf_counter() - t0) / repeats * 1e3
            ent = {"payload_bytes": nbytes, "alg_bytes_per_launch": alg,
                   "kernel_us": round(ms * 1e3, 2),
                   "roofline": {"bound": "hbm", "achieved": round(alg / (ms / 1e3) / 1e9, 1), "peak": peak,
                                "unit": "GB/s", "frac": round(alg / (ms / 1e3) / 1e9 / peak, 4),
                                "peak_kind": peak_kind},
                   "pack_e2e_ms": round(pack_ms, 3), "unpack_e2e_ms": round(unpack_ms, 3)}
            if mode != GFF_TERRAIN:
                t0 = time.perf_counter()
                O.pack(mode, f.uk, f.vk, f.wk, kkart=dom.static.kkart, dxk=dom.dxk)
                ent["cpu_pack_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
                ent["cpu_kind"] = "numpy restatement, 1 core"
            out["formats"][name] = ent
    return out


def prep_measure(dom, repeats: int = 5):
    """Set-up entry points on the grid of `dom` (rank 0 only)."""
    import numpy as np
    from gral_b200.abi import MetProfile
    from gral_b200.prognostic import PrognosticSolver
    from oracle import prep as OP

    F32 = np.float32
    st = dom.static
    th = math.radians(225.0)                 # the production situation: 225 deg, 2 m/s at 10 m, neutral
    met = MetProfile(np.array([0, 10.0], F32), np.array([0, -2.0 * math.sin(th)], F32),
                     np.array([0, -2.0 * math.cos(th)], F32), 1000.0)
    grid = dict(nii=dom.nii, njj=dom.njj, nkk=dom.nkk, vert_cells_ff=dom.vert_cells_ff, dxk=dom.dxk,
                dyk=dom.dyk, near_wall=0, igeb=max(int(20 / dom.dxk), 1))
    rng = np.random.default_rng(2)
    lines = [dict(crown_height=float(rng.uniform(2, 25)), trunk_height=float(rng.uniform(0, 8)),
                  trunk_lad=float(rng.uniform(0.05, 0.5)), crown_lad=float(rng.uniform(0.1, 1.5)),
                  cov=float(rng.uniform(0.1, 1.0)), i=int(rng.integers(1, dom.nii + 1)),
                  j=int(rng.integers(1, dom.njj + 1)), drag=1) for _ in range(20000)]
    cov0 = np.zeros((dom.nii + 2, dom.njj + 2), F32)
    peak, peak_kind = measured_peak()
    cols = dom.nii * dom.njj
    cells = cols * dom.nkk
    calls = {
        "subdomains": (lambda s: s.subdomains(st.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 15),
                       lambda: OP.subdomains(st.cutk, dom.nii, dom.njj, dom.dxk, dom.dyk, 15), None),
        # per column: CUTK read, KKART and AHK written; per level: U and V written
        "flat_init": (lambda s: s.flat_init(grid, st.cutk, st.dzk, st.hokart, met),
                      lambda: OP.flat_init(grid, st.cutk, st.dzk, st.hokart, met), 10 * cols + 8 * cells),
        "flat_init_near_wall": (lambda s: s.flat_init(dict(grid, near_wall=1), st.cutk, st.dzk, st.hokart, met,
                                                      st.advdom),
                                lambda: OP.flat_init(dict(grid, near_wall=1), st.cutk, st.dzk, st.hokart, met,
                                                     st.advdom), None),
        "vegetation_20k_lines": (lambda s: s.vegetation(dom.nii, dom.njj, dom.nkk, st.kkart, st.dzk, st.hokart,
                                                        lines, cov0),
                                 lambda: OP.vegetation(dom.nii, dom.njj, dom.nkk, st.kkart, st.dzk, st.hokart,
                                                       lines, cov0), None),
    }
    out = {"workload": f"{dom.nii}x{dom.njj}x{dom.nkk} city grid, production situation (225 deg, 2 m/s at 10 m)",
           "calls": {}}
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for name, (dev, cpu, alg) in calls.items():
            dev(s)
            ks, ts = [], []
            for _ in range(repeats):
                t0 = time.perf_counter()
                dev(s)
                ts.append(time.perf_counter() - t0)
                ks.append(s.prep_last_ms())
            t0 = time.perf_counter()
            cpu()
            cpu_ms = (time.perf_counter() - t0) * 1e3
            kms = statistics.median(ks)
            ent = {"kernel_ms": round(kms, 4), "call_ms": round(statistics.median(ts) * 1e3, 3),
                   "cpu_oracle_ms": round(cpu_ms, 1), "cpu_kind": "oracle restatement, 1 core"}
            if alg:
                ach = alg / (kms / 1e3) / 1e9
                ent["roofline"] = {"bound": "hbm", "alg_bytes_per_launch": alg, "achieved": round(ach, 1),
                                   "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": peak_kind}
            out["calls"][name] = ent
    return out


def batch_setup_measure(dom, n: int = 144, sample: int = 4):
    """Loading a batch of n situations: initial fields built on the device from met profiles
    (gral_prog_load_flat) against host-built fields copied in (gral_prog_load) (rank 0 only)."""
    import numpy as np
    from gral_b200.abi import FieldArrays, MetProfile
    from gral_b200.prognostic import PrognosticSolver
    from oracle import prep as OP

    F32 = np.float32
    st = dom.static
    grid = dict(nii=dom.nii, njj=dom.njj, nkk=dom.nkk, vert_cells_ff=dom.vert_cells_ff, dxk=dom.dxk,
                dyk=dom.dyk, near_wall=0, igeb=max(int(20 / dom.dxk), 1))
    mets = []
    for q in range(n):
        th = math.radians(10.0 * (q % 36))
        sp = (0.5, 1.0, 2.0, 4.0)[(q // 36) % 4]
        mets.append(MetProfile(np.array([0, 10.0], F32), np.array([0, -sp * math.sin(th)], F32),
                               np.array([0, -sp * math.cos(th)], F32), (250.0, 1000.0, -60.0)[q % 3]))
    ps = [dom.params(None, iterations=1) for _ in range(n)]
    shape = (dom.nii + 2, dom.njj + 2, dom.nkk + 2)
    out = FieldArrays(np.zeros(shape, F32), np.zeros(shape, F32), np.zeros(shape, F32))
    t0 = time.perf_counter()
    host = [OP.flat_init(grid, st.cutk, st.dzk, st.hokart, mets[q])[3] for q in range(sample)]
    host_s = (time.perf_counter() - t0) / sample * n
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=n) as s:
        s.load_flat(ps[:2], st, mets[:2], grid, [out, out])
        t0 = time.perf_counter()
        s.load_flat(ps, st, mets, grid, [out] * n)
        flat_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        s.load(ps, st, [host[q % sample] for q in range(n)])
        load_s = time.perf_counter() - t0
    return {"workload": f"{n} situations on the {dom.nii}x{dom.njj}x{dom.nkk} grid (met profiles of the batched set)",
            "load_flat_s": round(flat_s, 3), "load_host_fields_s": round(load_s, 3),
            "host_setup_s_estimate": round(host_s, 1),
            "host_setup_kind": f"oracle restatement of MicroscaleFlat.cs on 1 core, {sample} situations timed, scaled to {n}"}


def wind_measure(dom, sit, n: int = 1 << 20, repeats: int = 5):
    """Wind interpolation at n particles after a store (rank 0 only)."""
    import numpy as np
    from gral_b200 import prep
    from gral_b200.abi import PARTICLE_DTYPE
    from gral_b200.prognostic import PrognosticSolver
    from oracle import prep as OP

    f = prep.initial_fields(dom, sit)
    rng = np.random.default_rng(9)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["i"] = rng.integers(1, dom.nii + 1, n)
    p["j"] = rng.integers(1, dom.njj + 1, n)
    p["x"] = (p["i"] - 1) * dom.dxk + rng.uniform(0, dom.dxk, n)
    p["y"] = (p["j"] - 1) * dom.dyk + rng.uniform(0, dom.dyk, n)
    p["z"] = rng.uniform(0.0, 200.0, n).astype(np.float32)
    g = dict(terrain=0, buildings=1, ikooa=0, jkooa=0, dxk=dom.dxk, dyk=dom.dyk)
    st = dom.static
    peak, peak_kind = measured_peak()
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        s.load([dom.params(sit, iterations=1)], st, [f])
        s.store([f])
        s.wind_at(0, g, st.dzk, st.hokart, p)
        ks, ts = [], []
        for _ in range(repeats):
            t0 = time.perf_counter()
            s.wind_at(0, g, st.dzk, st.hokart, p)
            ts.append(time.perf_counter() - t0)
            ks.append(s.prep_last_ms())
    t0 = time.perf_counter()
    OP.wind_at(g, dom.nii, dom.njj, dom.nkk, st.dzk, st.hokart, f, p)
    cpu_s = time.perf_counter() - t0
    kms = statistics.median(ks)
    # per particle: its 32 B record, 16 B of results and six field values from random cells, each
    # of which moves a whole 32 B sector
    alg = (32 + 16 + 6 * 32) * n
    ach = alg / (kms / 1e3) / 1e9
    return {"workload": f"{n} random particles below 200 m on the {dom.nii}x{dom.njj}x{dom.nkk} field (flat, buildings)",
            "kernel_ms": round(kms, 4), "particles_per_s_kernel": round(n / (kms / 1e3), 0),
            "call_ms": round(statistics.median(ts) * 1e3, 3),
            "particles_per_s_call": round(n / statistics.median(ts), 0),
            "roofline": {"bound": "hbm", "alg_bytes_per_launch": alg, "achieved": round(ach, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(ach / peak, 4), "peak_kind": peak_kind},
            "cpu_oracle_particles_per_s": round(n / cpu_s, 0), "cpu_kind": "oracle restatement, 1 core"}


def instances_measure(n: int = 16, iterations: int = 100, concurrent: int = 16, seed: int = 0, distinct: int = 32):
    """Uneven-domain instances, sequential against side by side (rank 0 only).  Up to `distinct`
    grids are drawn (log-uniform 128..512 columns a side at 2-4 m, hills and buildings); instance q
    solves grid q % distinct with its own random inflow."""
    import numpy as np
    from gral_b200 import prep
    from gral_b200.prognostic import solve_instances

    rng = np.random.default_rng(seed)
    grids = []
    for q in range(min(n, distinct)):
        side = int(round(math.exp(rng.uniform(math.log(128), math.log(512)))))
        nj = int(round(side * rng.uniform(0.8, 1.0)))
        vc = int(round(20 + (side - 128) / (512 - 128) * 20))
        dx = float(rng.choice([2.0, 3.0, 4.0]))
        grids.append(prep.hilly_domain(side, nj, dx, vc, seed=100 + q))
    doms, ps, fs = [], [], []
    for q in range(n):
        d = grids[q % len(grids)]
        sit = prep.random_situation(100 + q)
        doms.append(d)
        ps.append(d.params(sit, model=1, iterations=iterations))
        fs.append(prep.initial_fields(d, sit))
    statics = [d.static for d in doms]
    cells = sum(int((d.static.advdom[1:d.nii + 1, 1:d.njj + 1] == 1).sum()) * d.vert_cells_ff for d in doms)
    out = {"workload": f"{n} instances on {len(grids)} grids of {min(d.nii for d in doms)}..{max(d.nii for d in doms)} "
                       f"columns a side, {iterations} iterations each, model 1", "cells": cells}
    for name, k in (("sequential", 1), ("side_by_side", concurrent)):
        f2 = [f.copy() for f in fs]
        t0 = time.perf_counter()
        _, status, rc = solve_instances(ps, statics, f2, max_concurrent=k)
        dt = time.perf_counter() - t0
        out[name] = {"max_concurrent": k, "seconds": round(dt, 3), "status_ok": rc == 0,
                     "value": round(cells * iterations / dt / 1e6, 3), "unit": UNIT,
                     "instances_per_hour_at_800_iterations": round(3600.0 * n / (dt * 800 / iterations), 1)}
    out["speedup"] = round(out["sequential"]["seconds"] / out["side_by_side"]["seconds"], 3)
    return out


def to_stop_measure(dom, batch: int = 144, max_iters: int = 800, threshold: float = 1e-3, plain_n: int = 1):
    """The weather-situation set solved to its stop rule (rank 0 only): each situation stops at
    _delta < threshold at a test every 100 iterations (from iteration 100) or at max_iters, as one
    batched solve through gral_prog_solve_batch, against plain single-situation solves of the first
    plain_n situations of the set (one call each); both host-timed end to end (fields in, set-up,
    iterations, post-checks, fields out), situations/hour measured, not extrapolated."""
    from gral_b200 import prep
    from gral_b200.prognostic import PrognosticSolver
    sits = batched_situations(batch)
    ps = [dom.params(x, model=1, iterations=max_iters, iter_min=100, conv_threshold=threshold) for x in sits]
    fs = [prep.initial_fields(dom, x) for x in sits]
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=batch) as s:
        t0 = time.perf_counter()
        sts = s.calculate_batch(ps, dom.static, fs)
        bt = time.perf_counter() - t0
    its = [x["iterations"] for x in sts]
    plain_s = []
    plain_its = []
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        for q in range(plain_n):
            f = prep.initial_fields(dom, sits[q])
            t0 = time.perf_counter()
            st = s.calculate(ps[q], dom.static, f)
            plain_s.append(time.perf_counter() - t0)
            plain_its.append(st["iterations"])
    per_plain = statistics.mean(plain_s)
    return {"workload": f"{batch} situations of the weather set on the {dom.nii}x{dom.njj}x{dom.vert_cells_ff} grid, "
                        f"stop at _delta < {threshold} (tested every 100 iterations) or {max_iters} iterations",
            "batched": {"seconds": round(bt, 3), "situations_per_hour": round(3600.0 * batch / bt, 1),
                        "iterations_min": min(its), "iterations_max": max(its),
                        "iterations_mean": round(statistics.mean(its), 1),
                        "converged": int(sum(x["converged"] for x in sts))},
            "plain": {"situations_timed": plain_n, "seconds_per_situation": round(per_plain, 3),
                      "iterations": plain_its, "situations_per_hour": round(3600.0 / per_plain, 1)},
            "batched_over_plain": round((3600.0 * batch / bt) / (3600.0 / per_plain), 3),
            "note": "one GPU; the plain form's situations/hour assumes the timed situations are representative "
                    "(same stop rule; every situation of the set ran to the same limit when none converged)"}


def adjoint_measure(iterations: int = 200, every: int = 20, n: int = 200):
    """The discrete adjoint on the differentiation workload (rank 0 only): a 200x200 grid at 2 m
    with 25 prognostic levels, 30 buildings, vegetation drag over 20 % of the columns, J = sum over
    1000 seeded probe cells of |(U, V, W) - target|^2 after 200 iterations, checkpoints every 20."""
    import numpy as np
    from gral_b200 import prep
    from gral_b200.prognostic import PrognosticSolver

    dom = prep.adjoint_domain(n)
    sit = prep.Situation(direction_deg=250.0, speed_10m=2.0, z0=0.3)
    f0 = prep.initial_fields(dom, sit)
    p = dom.params(sit, model=1, iterations=iterations, quantise=0)
    with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax) as s:
        fr = f0.copy()
        s.load([p], dom.static, [fr])               # the plain solve of the same map: fused launches
        s.iterate_timed(3)
        plain_ms, _ = s.iterate_timed(iterations - 3)
        plain_ms *= iterations / (iterations - 3)
        f = f0.copy()
        s.vjp_forward(p, dom.static, f, iterations, every)
        idx, tgt = prep.probe_misfit(dom, f, n_probes=1000, seed=11)
        J, g = prep.misfit_and_cotangent(idx, tgt, f.uk, f.vk, f.wk, np.float32)
        d_veg, d_uk0, d_vk0, d_wk0, st = s.vjp(*g)
        d_veg, d_uk0, d_vk0, d_wk0, st = s.vjp(*g)   # second call timed (first one pays the allocations)
        # every iteration's states kept on the device by the forward: nothing recomputed
        fa = f0.copy()
        s.vjp_forward(p, dom.static, fa, iterations, 0)
        s.vjp(*g)
        ga = s.vjp(*g)
        sta = ga[4]
        keep_all = {"forward_ms": round(sta["ms_forward"], 2), "vjp_ms": round(sta["ms_total"], 2),
                    "reverse_ms": round(sta["ms_reverse"], 2),
                    "cost_multiple_of_forward": round((sta["ms_forward"] + sta["ms_total"]) / sta["ms_forward"], 3),
                    "cost_multiple_of_checkpointed_forward": round((sta["ms_forward"] + sta["ms_total"]) / st["ms_forward"], 3),
                    "kept_bytes": int(iterations * 10 * (dom.nii + 2) * (dom.njj + 2) * ((dom.kadvmax + 9) // 8 * 8) * 4),
                    "grad_rel_l2_vs_checkpointed": float(np.linalg.norm(ga[0] - d_veg) / max(np.linalg.norm(d_veg), 1e-30))}
    inflow = prep.inflow_gradient(dom, sit, d_uk0.astype(np.float64), d_vk0.astype(np.float64))
    fwd = st["ms_forward"]
    return {"workload": f"{n}x{n}x{dom.vert_cells_ff} at 2 m, {len(dom.buildings)} buildings, VEG over "
                        f"{float(dom.static.veg_mask[1:n + 1, 1:n + 1].mean()):.2f} of the columns, 1000 probes, "
                        f"{iterations} iterations, checkpoints every {every}",
            "J": J, "iterations": iterations, "checkpoint_every": every,
            "forward_ms": round(fwd, 2), "plain_solve_ms": round(plain_ms, 2),
            "vjp_ms": round(st["ms_total"], 2), "recompute_ms": round(st["ms_recompute"], 2),
            "reverse_ms": round(st["ms_reverse"], 2),
            "cost_multiple_of_forward": round((fwd + st["ms_total"]) / fwd, 3),
            "cost_multiple_of_plain_solve": round((fwd + st["ms_total"]) / plain_ms, 3),
            "grad_norm_veg": float(np.linalg.norm(d_veg)), "dJ_dinflow": inflow, "keep_all": keep_all,
            "checks": "GPU gradients against FP64 central differences (20 directions, 32x32, 20 iterations) and "
                      "the FP64 tape gradient in tests/test_adjoint_gpu.py"}


def run_ours(args, rank, world):
    import torch
    from gral_b200 import prep
    from gral_b200.prognostic import PrognosticSolver

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = world > 1
    if dist:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    dom, sit, full_iters, desc = workload(args.workload, args.grid)
    sits = rank_situations(sit, args.batch, rank, world)
    nsit = len(sits)
    cells = nominal_cells(dom) * nsit
    t_max, _, phases, st_store, clocks = device_run(dom, sits, args.steps, args.warmup, local)
    value = cells * args.steps * world / (t_max / 1e3) / 1e6
    ms_per_step = t_max / args.steps
    layout = "interleaved" if st_store["layout"] == 1 else "slab"

    # end to end through the public ABI: pinned host buffers, full solve, fields back
    e2e = None
    if not args.no_e2e:
        e2e_iters = args.e2e_iters if args.e2e_iters > 0 else full_iters
        pes = [dom.params(x, model=1, iterations=e2e_iters, iter_min=e2e_iters) for x in sits]
        fps = [pinned_fields(prep.initial_fields(dom, x)) for x in sits]
        with PrognosticSolver(dom.nii, dom.njj, dom.nkk, dom.kadvmax, max_batch=nsit) as s2:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sts = s2.calculate_batch(pes, dom.static, fps)
            dt = time.perf_counter() - t0
        iters = sum(x["iterations"] for x in sts) / nsit
        dt = max_over_ranks(dt, "cuda")
        nbytes = sum(a.nbytes for fp in fps for a in (fp.uk, fp.vk, fp.wk))
        e2e = {"value": round(cells * iters * world / dt / 1e6, 3), "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "iterations": iters, "seconds": round(dt, 4),
               "situations_per_hour": round(3600.0 * nsit * world / dt, 1),
               "note": "one step = one full solve (set-up, all iterations, post-checks, fields back)"}

    # the batched form beside the plain one (same grid, 144 situations), device-timed
    batched = None
    if args.workload == "production" and not args.no_batched:
        bsits = rank_situations(None, args.batch, rank, world)
        bcells = nominal_cells(dom) * len(bsits)
        bt, _, bph, bst, bclk = device_run(dom, bsits, args.batched_steps, 3, local)
        bms = bt / args.batched_steps
        batched = {"workload": f"batched: {len(bsits)} situations on the same grid", "situations": len(bsits),
                   "value": round(bcells * args.batched_steps * world / (bt / 1e3) / 1e6, 3), "unit": UNIT,
                   "steps": args.batched_steps, "warmup": 3, "ms_per_step": round(bms, 4),
                   "layout": "interleaved" if bst["layout"] == 1 else "slab",
                   "launch_variant": bst["launch_variant"],
                   "gpu_launches": bst["launches_per_iteration"] * args.batched_steps,
                   "situations_per_hour_at_800_iterations": round(3600.0 * len(bsits) * world / (bms * 800 / 1e3), 1),
                   "roofline": roofline(bcells, args.batched_steps, bph,
                                        "interleaved" if bst["layout"] == 1 else "slab"),
                   "phase_ms_per_iteration": {k: round(v / args.batched_steps, 4) for k, v in bph.items() if v > 0},
                   "clocks": bclk}

    # the weather set solved to its stop rule, batched against plain (single GPU)
    tostop = None
    if args.workload == "production" and rank == 0 and world == 1 and not args.no_batched and not args.no_to_stop:
        tostop = to_stop_measure(dom, args.batch)
        if batched is not None:
            batched["to_stop"] = tostop

    # the measurements of the rows around the solve run on single-GPU runs only
    extras = rank == 0 and world == 1 and args.workload == "production"
    gffm = None
    if extras and not args.no_gff:
        gffm = gff_measure(dom, sit)
    prepm = None
    if extras and not args.no_prep:
        prepm = prep_measure(dom)
        prepm["batch_setup"] = batch_setup_measure(dom)
    windm = None
    if extras and not args.no_wind:
        windm = wind_measure(dom, sit)
    instm = None
    if extras and not args.no_instances:
        instm = instances_measure(args.instances, args.instances_iters, args.instances_concurrent)
    adjm = None
    if extras and not args.no_adjoint:
        adjm = adjoint_measure(args.adjoint_iters, args.adjoint_every)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = CpuBaseline(args.workload, args.cpu_iters)
        try:
            cpu = cb.describe(*cb.step())
        finally:
            cb.close()

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "cells": cells, "situations": nsit,
                   "grid": [dom.nii, dom.njj, dom.nkk], "kadvmax": dom.kadvmax, "model": 1,
                   "simd_parity_width": 8, "l2": "inputs larger than L2 (8 fields x 31 MB per situation)",
                   "parallelism": (f"replicas x{world}" if sit is not None else f"situations sharded x{world}"),
                   "layout": layout, "launch_variant": st_store["launch_variant"]},
        "phase_ms_per_iteration": {k: round(v / args.steps, 4) for k, v in phases.items() if v > 0},
        "roofline": roofline(cells, args.steps, phases, layout),
        "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": st_store["launches_per_iteration"] * args.steps,
        "clocks": clocks,
        "gff": gffm, "prep": prepm, "wind": windm, "instances": instm, "adjoint": adjm,
        # last on the line, so that a reader keeping only the end of the line still has it
        "batched": batched,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        td.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["production", "batched", "cube"], default="production")
    ap.add_argument("--batch", type=int, default=144, help="situations of the batched workload")
    ap.add_argument("--grid", type=int, default=400, help="columns per side of the city grid (profiling cases)")
    ap.add_argument("--e2e-iters", type=int, default=0, help="iterations of the e2e solve (0: the workload's)")
    ap.add_argument("--cpu-iters", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched sub-measurement")
    ap.add_argument("--batched-steps", type=int, default=10)
    ap.add_argument("--no-gff", action="store_true", help="skip the flow-field cache payload measurement")
    ap.add_argument("--no-prep", action="store_true", help="skip the set-up (sub-domains, initial field) measurement")
    ap.add_argument("--no-wind", action="store_true", help="skip the particle wind interpolation measurement")
    ap.add_argument("--no-instances", action="store_true", help="skip the uneven-domain instances measurement")
    ap.add_argument("--instances", type=int, default=16, help="instances of the uneven-domain measurement")
    ap.add_argument("--instances-iters", type=int, default=100, help="SIMPLE iterations per uneven-domain instance")
    ap.add_argument("--instances-concurrent", type=int, default=16, help="slots of the packed uneven-domain run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint measurement")
    ap.add_argument("--adjoint-iters", type=int, default=200, help="unrolled iterations of the adjoint measurement")
    ap.add_argument("--adjoint-every", type=int, default=20, help="checkpoint spacing of the adjoint measurement")
    ap.add_argument("--no-to-stop", action="store_true", help="skip the weather set solved to its stop rule")
    ap.add_argument("--ref-iters", type=int, default=4, help="SIMPLE iterations per reference-arm step")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
