#!/usr/bin/env python
"""Benchmark of the B200 octree-AMR lattice Boltzmann time step.

One "step" is one coarse time step of the solver (Mesh::M_Advance_Step: the
S_Advance recursion from N_LEVEL_START over every level, plus the
solution-based refinement when its P_REFINE turn comes) on the workload named
in the JSON line.  Metric: MLUPS, million lattice-cell updates per second,
leaf cells of level L counted 2^(L-L0) times per coarse step as
solver_lbm_advance.cu:74-89 counts them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Default workload: D2Q9 lid-driven cavity on a 128^2 base grid with up to 3
levels, refined above the 90th and coarsened below the 50th percentile of the
block vorticity every 64 coarse steps, Re = 1000, lid 0.05, FP16 weight-offset
populations.  The multi-level hierarchy is developed by an untimed spin-up
before the warm-up.  The same case in FP32 populations is timed beside it
(`plain_fp32`).

--impl b200 (default): the CUDA library.  Rank 0 prints one JSON line with
  value        device-timed MLUPS (CUDA events on the library's stream, L2
               flushed between steps when the state fits in L2)
  e2e          MLUPS through the public C ABI with host buffers: load the
               populations from pinned host memory, K x (coarse step + read
               back the FP64 mass/momentum), dump the populations
  roofline     the fused step kernel on a large single-level case of the same
               physics and storage (inputs far larger than L2), algorithmic
               bytes 2*Q*s per cell update
  cpu_baseline the CPU oracle (OpenMP restatement of the reference algorithm)
               on a bounded sample of the same workload, rank 0 only
--impl reference: the reference's algorithm on the host cores (the CPU oracle
  port; the reference has no CPU implementation of its own), rank 0 only.

Multi-GPU: one process per GPU under torchrun; every rank runs an
independent replica of the workload (a single case does not shard), so the
scaling is weak and `value` is the sum over ranks divided by the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import agal_b200 as ag  # noqa: E402
from agal_b200 import _lib  # noqa: E402

L2_BYTES = 126 * 2 ** 20

_AMR = dict(amr=True, levels=3, p_refine=64, Re=1000.0, bc=_lib.BC_LDC2D, velocity_set=_lib.D2Q9, Nx=128,
            interp=_lib.INTERP_CUBIC, spinup=1280)
# Workloads (synthetic: initialised at rest, nothing read from disk).
WORKLOADS = {
    "amr_ldc2d_128_fp16": dict(
        _AMR, storage=_lib.STORE_FP16,
        desc="D2Q9 BGK lid-driven cavity, 128^2 base in 4^2-cell blocks, up to 3 levels, percentile vorticity "
             "criterion (refine > p90, coarsen < p50) every 64 coarse steps, Re=1000, lid 0.05, cubic "
             "interpolation, FP16 weight-offset populations"),
    "amr_ldc2d_128": dict(
        _AMR, storage=_lib.STORE_FP32,
        desc="D2Q9 BGK lid-driven cavity, 128^2 base in 4^2-cell blocks, up to 3 levels, percentile vorticity "
             "criterion (refine > p90, coarsen < p50) every 64 coarse steps, Re=1000, lid 0.05, cubic "
             "interpolation, FP32 populations"),
    "ldc2d_256": dict(
        desc="D2Q9 BGK lid-driven cavity 256x256, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=256, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_256_fp16": dict(
        desc="D2Q9 BGK lid-driven cavity 256x256, one level, Re=100, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D2Q9, Nx=256, Re=100.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC2D),
    "ldc2d_4096": dict(
        desc="D2Q9 BGK lid-driven cavity 4096x4096, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=4096, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_4096_fp16": dict(
        desc="D2Q9 BGK lid-driven cavity 4096x4096, one level, Re=100, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D2Q9, Nx=4096, Re=100.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC2D),
    "ldc2d_8192": dict(
        desc="D2Q9 BGK lid-driven cavity 8192x8192, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=8192, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_8192_fp16": dict(
        desc="D2Q9 BGK lid-driven cavity 8192x8192, one level, Re=100, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D2Q9, Nx=8192, Re=100.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC2D),
    "ldc3d19_384": dict(
        desc="D3Q19 BGK lid-driven cavity 384^3, one level, Re=400, lid 0.05, FP32 populations",
        velocity_set=_lib.D3Q19, Nx=384, Re=400.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC3D),
    "ldc3d19_384_fp16": dict(
        desc="D3Q19 BGK lid-driven cavity 384^3, one level, Re=400, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D3Q19, Nx=384, Re=400.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC3D),
    "ldc3d27_256": dict(
        desc="D3Q27 BGK lid-driven cavity 256^3, one level, Re=200, lid 0.05, FP32 populations",
        velocity_set=_lib.D3Q27, Nx=256, Re=200.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC3D),
}
Q_OF = {_lib.D2Q9: 9, _lib.D3Q19: 19, _lib.D3Q27: 27}
DIM_OF = {_lib.D2Q9: 2, _lib.D3Q19: 3, _lib.D3Q27: 3}
ESIZE = {_lib.STORE_FP32: 4, _lib.STORE_FP64: 8, _lib.STORE_FP16: 2, _lib.STORE_BF16: 2}
DTYPE_NAME = {_lib.STORE_FP32: "f32", _lib.STORE_FP64: "f64", _lib.STORE_FP16: "f16-offset(f32 math)",
              _lib.STORE_BF16: "bf16-offset(f32 math)"}
ROOFLINE_FOR = {_lib.STORE_FP16: "ldc2d_8192_fp16", _lib.STORE_FP32: "ldc2d_8192"}


def make_params(w: dict, device: int = -1):
    dim = DIM_OF[w["velocity_set"]]
    nb = (w["Nx"] // 4) ** dim
    kw = dict(velocity_set=w["velocity_set"], Nx=w["Nx"], MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1,
              N_LEVEL_START=0, v0=0.05 / w["Re"], bc_preset=w["bc"], ic_preset=_lib.IC_REST,
              storage=w["storage"], n_maxcblocks=nb, device=device)
    if w.get("amr"):
        nch = 2 ** dim
        kw.update(MAX_LEVELS_INTERIOR=w["levels"], P_REFINE=w["p_refine"], S_CRITERION=_lib.CRITERION_PERCENTILE,
                  ref_pct_hi=0.9, ref_pct_lo=0.5, interp_order=w["interp"],
                  n_maxcblocks=sum(nb * nch ** L for L in range(w["levels"])) + 64)
    return ag.default_params(**kw)


def leaf_cells(counts: dict, dim: int) -> int:
    """Cell updates of one coarse step (solver_lbm_advance.cu:74-89): leaf
    blocks of level L, counted 2^L times, times the cells per block."""
    n = counts["n_ids"]
    ml = counts["max_levels"]
    nch, mc = 2 ** dim, 4 ** dim
    cells = 0
    for L in range(ml):
        leaves = n[L] - (n[L + 1] // nch if L + 1 < ml else 0)
        cells += (1 << L) * leaves
    return cells * mc


def state_bytes(case, w: dict) -> int:
    c = case.counts()
    return sum(c["n_ids"][: c["max_levels"]]) * 4 ** DIM_OF[w["velocity_set"]] * Q_OF[w["velocity_set"]] * \
        ESIZE[w["storage"]]


def launches_per_step(counts: dict, amr: bool) -> int:
    """Kernels of one coarse step, from the structure of the level recursion:
    level L takes 2^L sub-steps, each a fused step and its stream-guard
    fix-up, and every non-empty level below the finest launches 2^L
    interpolations and 2^L averagings."""
    if not amr:
        return 2
    n, ml = counts["n_ids"], counts["max_levels"]
    total = 0
    for L in range(ml):
        if n[L] == 0:
            continue
        mult = 1 << L
        total += 2 * mult
        if L < ml - 1:
            total += 2 * mult
    return total


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock/throttle samples taken while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self) -> dict:
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}




def measured_peak_hbm() -> tuple[float, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def dram_traffic_per_launch(workload: str):
    """DRAM bytes per launch of the fused step kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "k_step_traffic.json"
    if not f.exists():
        return None
    try:
        d = json.loads(f.read_text())
        return d.get(workload, {}).get("dram_bytes_per_launch")
    except ValueError:
        return None


# ---------------------------------------------------------------------------
def step_fn(case, w: dict):
    """One coarse step: the captured multi-level step (with its regrid turn)
    or the fused single-level step."""
    if w.get("amr"):
        return lambda: case.advance_n(1, use_graph=True)
    return case.advance


def time_steps(case, torch, w: dict, n_steps: int, flush: bool):
    """Per-step device time (ms) with CUDA events on the library's stream,
    and the cell updates of each step."""
    stream = torch.cuda.ExternalStream(case.stream_ptr())
    scratch = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda") if flush else None
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
    step = step_fn(case, w)
    dim = DIM_OF[w["velocity_set"]]
    cells, launches = [], 0
    for i in range(n_steps):
        if flush:
            with torch.cuda.stream(stream):
                scratch.add_(1.0)   # writes 252 MB > L2 between timed steps
        cnt = case.counts()
        cells.append(leaf_cells(cnt, dim))
        launches += launches_per_step(cnt, w.get("amr", False))
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    case.sync()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs], cells, launches


def develop(case, w: dict):
    """Initial state, then the untimed spin-up that builds the hierarchy."""
    case.set_ic(0)
    if w.get("amr"):
        case.refine_near_wall()
        case.advance_n(w["spinup"], use_graph=True)


# ---------------------------------------------------------------------------
# Batched workload: many independent D3Q19 cases advanced together
# (agal_batch: one CUDA graph per coarse step, one branch per case) against
# the same cases in FP32, one at a time.
BATCH_SIZES = (32, 48, 64, 96)


def batched_specs(n: int, seed: int) -> list[dict]:
    """Seeded case list: base N^3 with N in {32, 48, 64, 96}, 1-3 levels, Re
    log-uniform in [100, 1000] (on the unit domain length, v0 = 0.05/Re), half
    lid-driven cavities (solution refinement, percentile criterion), half flow
    past a seeded random ellipsoid (axes 8-24 cells, near-wall refinement,
    interpolated bounce-back, MEA forces)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        s = dict(N=int(rng.choice(BATCH_SIZES)), levels=int(rng.integers(1, 4)),
                 Re=float(np.exp(rng.uniform(np.log(100.0), np.log(1000.0)))),
                 kind="cavity" if i % 2 == 0 else "ellipsoid")
        if s["kind"] == "ellipsoid":
            s["axes"] = [float(a) for a in rng.uniform(8.0, 24.0, size=3)]
            s["centre"] = [float(x) for x in rng.uniform(0.42, 0.58, size=3)]
            s["seed"] = int(rng.integers(1 << 30))
        out.append(s)
    return out


def batched_case(s: dict, storage: int, device: int):
    from agal_b200.geometry import icosphere
    N, lv = s["N"], s["levels"]
    nb = (N // 4) ** 3
    kw = dict(velocity_set=_lib.D3Q19, Nx=N, v0=0.05 / s["Re"], storage=storage, device=device,
              interp_order=_lib.INTERP_LINEAR, P_REFINE=32, S_CRITERION=_lib.CRITERION_PERCENTILE,
              ref_pct_hi=0.9, ref_pct_lo=0.5, n_maxcblocks=nb if lv == 1 else 3 * nb + 2048)
    if s["kind"] == "cavity":
        kw.update(MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=lv, bc_preset=_lib.BC_LDC3D, ic_preset=_lib.IC_REST)
    else:
        kw.update(MAX_LEVELS_WALL=lv, MAX_LEVELS_INTERIOR=1, bc_preset=_lib.BC_FPSC3D, ic_preset=_lib.IC_UNIFORM,
                  u_ref=0.05, G_BIN_DENSITY=8, G_BIN_LEVELS=lv, G_BIN_SPEC=2, G_BIN_MAKE_LINKS=1,
                  G_NEAR_WALL_DISTANCE=0.05, S_BC_TYPE=1, S_FORCE_TYPE=0, S_FORCE_ORDER=2)
    case = ag.Case(ag.default_params(**kw))
    if s["kind"] == "ellipsoid":
        # Axes in cells of the base grid, at most half the base size, so that
        # the body and its refinement band stay clear of the domain faces.
        axes = np.minimum(np.asarray(s["axes"]), 0.5 * N)
        f = icosphere(3, 1.0, (0.0, 0.0, 0.0), seed=s["seed"]).astype(np.float64)
        f = f * (axes / (2.0 * N)) + np.asarray(s["centre"])
        case.set_geometry(f.astype(np.float32))
    case.set_ic(0)
    case.refine_near_wall()
    return case


def run_batched(torch, n_cases: int, seed: int, spinup: int, steps: int, device: int) -> dict:
    """Aggregate MLUPS of the batch (FP16 populations, batched graph) and of
    the same cases in FP32 advanced one at a time; both after the same
    spin-up, timed with CUDA events over `steps` coarse steps that hold no
    regrid (P_REFINE = 32, spin-up past the first regrid)."""
    specs = batched_specs(n_cases, seed)

    def build(storage):
        cases = [batched_case(s, storage, device) for s in specs]
        tunes = [c.autotune(0, reps=3)["variant"] for c in cases]
        return cases, tunes

    def cells(cases):
        return sum(leaf_cells(c.counts(), 3) for c in cases)

    # batched, FP16
    cases, tunes16 = build(_lib.STORE_FP16)
    batch = ag.Batch(cases)
    batch.advance_n(spinup)
    batch.sync()
    stream = torch.cuda.ExternalStream(batch.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    upd16 = cells(cases)
    torch.cuda.synchronize()
    e0.record(stream)
    batch.advance_n(steps)
    e1.record(stream)
    batch.sync()
    t16 = e0.elapsed_time(e1)
    levels16 = [c.counts()["n_ids"][:-1] for c in cases]
    batch.close()
    for c in cases:
        c.close()
    # one at a time, FP32
    cases, tunes32 = build(_lib.STORE_FP32)
    for c in cases:
        c.advance_n(spinup)
    t32 = 0.0
    upd32 = cells(cases)
    for c in cases:
        c.sync()
        st = torch.cuda.ExternalStream(c.stream_ptr())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        c.advance_n(steps)
        b.record(st)
        c.sync()
        t32 += a.elapsed_time(b)
    for c in cases:
        c.close()
    v16 = upd16 * steps / (t16 * 1e-3) / 1e6
    v32 = upd32 * steps / (t32 * 1e-3) / 1e6
    peak, kind = measured_peak_hbm()
    gbs = upd16 * steps * 2 * 19 * 2 / (t16 * 1e-3) / 1e9
    return {"workload": "batched_d3q19_64", "n_cases": n_cases, "seed": seed,
            "desc": "independent D3Q19 BGK cases, base N^3 with N in {32,48,64,96}, 1-3 levels, Re log-uniform "
                    "[100,1000], half lid-driven cavities with percentile solution refinement, half flow past "
                    "a seeded ellipsoid (axes 8-24 cells) with near-wall refinement, interpolated bounce-back "
                    "and MEA forces; refinement by the plain criterion (no learned predictor)",
            "spinup_steps": spinup, "timed_steps": steps,
            "value": v16, "unit": "MLUPS", "storage": "f16-offset", "ms_per_step": t16 / steps,
            "cell_updates_per_step": upd16,
            "one_at_a_time_fp32": {"value": v32, "ms_per_step": t32 / steps, "cell_updates_per_step": upd32},
            "ratio_vs_one_at_a_time_fp32": v16 / v32,
            "hbm": {"achieved_gbs": gbs, "peak": peak, "frac": gbs / peak, "peak_source": kind,
                    "bytes_per_update": 2 * 19 * 2},
            "autotune_variants": {"fp16": tunes16, "fp32": tunes32},
            "blocks_per_level_fp16": levels16}


def run_cpu_oracle(w: dict, seconds: float, threads: int, max_steps: int | None = None) -> dict:
    """Oracle (CPU restatement, OpenMP) MLUPS on a bounded sample of the workload."""
    from oracle.orc import OracleCase, build  # CPU baseline leg only
    build()
    p = make_params(w)
    o = OracleCase(p, p.n_maxcblocks, fp64=(w["storage"] == _lib.STORE_FP64), threads=threads)
    dim = DIM_OF[w["velocity_set"]]
    o.set_ic(0)
    spin = 0
    if w.get("amr"):
        o.refine_near_wall()
        spin = w["spinup"]
        o.advance_n(spin)
    t0 = time.perf_counter()
    o.advance_n(2)
    per = (time.perf_counter() - t0) / 2
    n = max(1, int(seconds / max(per, 1e-9)))
    if max_steps:
        n = min(n, max_steps)
    cells = 0
    t0 = time.perf_counter()
    for _ in range(n):
        cells += leaf_cells(o.counts(), dim)
        o.advance_n(1)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": cells / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{n} coarse steps of {w['desc']}" + (f" after a {spin}-step spin-up" if spin else "") +
                      f", on {threads} host threads ({dt:.1f} s)"}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def regrid_launches(counts: dict) -> int:
    """Kernels of one solution-based refinement, approximately: per parent
    level a refresh and a grid average, a refresh and an interface
    interpolation; the percentile criterion (block maxima, 4 x 2 selection
    passes, marks); about 40 in the refine/coarsen pass."""
    ml = counts["max_levels"]
    return 4 * (ml - 1) + 10 + 40


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="amr_ldc2d_128_fp16", choices=sorted(WORKLOADS))
    ap.add_argument("--plain-workload", default="amr_ldc2d_128", choices=sorted(WORKLOADS),
                    help="the same case in plain FP32, timed beside the headline workload")
    ap.add_argument("--roofline-workload", default=None, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--profile", choices=sorted(WORKLOADS), default=None,
                    help="only run W+K steps of this workload (for ncu captures); prints no JSON line")
    ap.add_argument("--cpt", type=int, default=1, choices=[1, 2, 3, 4, 5],
                    help="with --profile: step kernel variant (1, 2 cells per thread; 3 TMA pipeline; "
                         "4 one row of four cells per thread; 5 root-level tiles, 2D)")
    ap.add_argument("--batched-cases", type=int, default=64,
                    help="independent D3Q19 cases of the batched measurement (0 skips it)")
    ap.add_argument("--batched-seed", type=int, default=2024)
    ap.add_argument("--spinup", type=int, default=None,
                    help="with --profile: coarse steps of the untimed spin-up of a multi-level workload")
    a = ap.parse_args(argv)
    a.warmup = max(a.warmup, 3)
    w = WORKLOADS[a.workload]
    if a.profile:
        pw = dict(WORKLOADS[a.profile])
        if a.spinup is not None and pw.get("amr"):
            pw["spinup"] = a.spinup
        with ag.Case(make_params(pw, device=0)) as pc:
            develop(pc, pw)
            pc.set_tuning(a.cpt)
            step = step_fn(pc, pw)
            for _ in range(a.warmup + a.steps):
                step()
            pc.sync()
        print(f"profile run done: {a.profile}, {a.warmup}+{a.steps} steps")
        return 0
    ws, rank, local = dist_setup()
    threads = os.cpu_count() or 1
    base = {"metric": "MLUPS (lattice cell updates per second / 1e6), one coarse time step per step",
            "unit": "MLUPS", "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE_NAME[w["storage"]], "data": "synthetic (fluid at rest, lid-driven)"}

    def config_of(wl: str, extra: dict) -> dict:
        ww = WORKLOADS[wl]
        cfg = {"workload": wl, "desc": ww["desc"]}
        if ww.get("amr"):
            cfg.update(base_grid=f"{ww['Nx']}^2", levels=ww["levels"], regrid_every=ww["p_refine"],
                       spinup_steps=ww["spinup"])
        cfg.update(extra)
        return cfg

    if a.impl == "reference":
        # The reference algorithm on the host cores; other ranks idle.
        if rank != 0:
            return 0
        cb = run_cpu_oracle(w, seconds=1e9, threads=threads, max_steps=a.steps)
        line = dict(base, impl="reference", value=cb["value"], ms_per_step=None,
                    config=config_of(a.workload, {"parallelism": "host OpenMP", "l2": "n/a (CPU)"}),
                    cpu_baseline=cb, e2e={"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0})
        line["n_gpus"] = 0
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if ws > 1:
            dist.barrier()

    def allmax(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def device_timed(wl: str, with_clocks: bool):
        ww = WORKLOADS[wl]
        case = ag.Case(make_params(ww, device=local))
        develop(case, ww)
        tune = case.autotune(0, reps=10)
        step = step_fn(case, ww)
        for _ in range(a.warmup):
            step()
        case.sync()
        flush = state_bytes(case, ww) * 2 < L2_BYTES
        barrier()
        torch.cuda.synchronize()
        it0 = case.refine_stats()["iter"]
        if with_clocks:
            with ClockSampler(local) as clk:
                per_step, cells, launches = time_steps(case, torch, ww, a.steps, flush)
            clocks = clk.summary()
        else:
            per_step, cells, launches = time_steps(case, torch, ww, a.steps, flush)
            clocks = None
        if ww.get("amr"):
            p_ref = ww["p_refine"]
            regrids = sum(1 for i in range(it0, it0 + a.steps) if (i + 1) % p_ref == 0 and i > 0)
            launches += regrids * regrid_launches(case.counts())
        counts = case.counts()
        barrier()
        t_ms = allmax(sum(per_step))
        mlups = allsum(float(sum(cells))) / (t_ms * 1e-3) / 1e6
        case.close()
        return dict(value=mlups, ms_per_step=t_ms / a.steps, flush=flush, tune=tune, clocks=clocks,
                    launches=launches, counts=counts, cells_per_step=float(np.mean(cells)))

    def learned_timed(wl: str, wl_src: str):
        """The workload with the learned predictor driving its refinement: the
        network is trained on the GPU on snapshots of the plain FP32 run's
        spin-up (labelled by the percentile rule), then predicts the marks of
        every regrid of a fresh run, the rule judging every 4th regrid."""
        ww, ws_ = WORKLOADS[wl], WORKLOADS[wl_src]
        dim = DIM_OF[ww["velocity_set"]]
        t0 = time.perf_counter()
        src = ag.Case(make_params(ws_, device=local))
        m = ag.Learner(dim, seed=7)
        m.attach(src, 1)
        develop(src, ws_)
        src.sync()
        nl = m.counts()["labelled"]
        weights = m.balance_classes(0, nl)
        loss = m.train(0, nl, 40, lr=2e-3, seed=7)
        thr = m.calibrate_thresholds(0, nl)
        m.attach(src, 0)
        src.close()
        train_s = time.perf_counter() - t0
        case = ag.Case(make_params(ww, device=local))
        m.attach(case, 2, judge_every=4)
        m.set_thresholds(*thr)
        develop(case, ww)
        tune = case.autotune(0, reps=10)
        step = step_fn(case, ww)
        for _ in range(a.warmup):
            step()
        case.sync()
        flush = state_bytes(case, ww) * 2 < L2_BYTES
        c0 = m.counts()
        barrier()
        torch.cuda.synchronize()
        per_step, cells, launches = time_steps(case, torch, ww, a.steps, flush)
        c1 = m.counts()
        counts = case.counts()
        barrier()
        t_ms = allmax(sum(per_step))
        mlups = allsum(float(sum(cells))) / (t_ms * 1e-3) / 1e6
        m.attach(case, 0)
        case.close()
        m.close()
        return dict(workload=wl, value=mlups, ms_per_step=t_ms / a.steps, snapshots=nl, class_weights=weights,
                    train_loss=loss, thresholds=thr, collect_and_train_s=train_s,
                    regrids=c1["regrids"] - c0["regrids"], judged=c1["judged"] - c0["judged"],
                    plain_refine_marks=c1["plain_refine"] - c0["plain_refine"],
                    missed=c1["missed"] - c0["missed"], blocks_per_level=counts["n_ids"][:-1],
                    cell_updates_per_step=float(np.mean(cells)), tune=tune)

    # --- device-timed steps: headline workload, then the plain FP32 form -------
    head = device_timed(a.workload, with_clocks=True)
    learned = learned_timed(a.workload, a.plain_workload) if WORKLOADS[a.workload].get("amr") else None
    plain = device_timed(a.plain_workload, with_clocks=False) if a.plain_workload != a.workload else None

    # --- end to end through the C ABI with host buffers ----------------------
    case = ag.Case(make_params(w, device=local))
    develop(case, w)
    case.set_tuning(head["tune"]["variant"])
    f0 = case.dump(_lib.ARR_F)
    pinned = torch.from_numpy(f0).pin_memory()
    host_in = pinned.numpy()
    host_out = torch.empty_like(pinned).pin_memory().numpy()
    mm = (C.c_double * 4)()
    lib = _lib.lib()
    dim = DIM_OF[w["velocity_set"]]
    amr = bool(w.get("amr"))
    e2e_cells = 0
    barrier()
    t0 = time.perf_counter()
    rc = lib.agal_load(case._h, _lib.ARR_F, host_in.ctypes.data_as(C.c_void_p), host_in.nbytes)
    for _ in range(a.steps):
        e2e_cells += leaf_cells(case.counts(), dim)
        rc |= lib.agal_advance_n(case._h, 1, 1) if amr else lib.agal_advance(case._h, 0)
        rc |= lib.agal_mass_momentum(case._h, mm)   # D2H of the step's FP64 mass/momentum
    rc |= lib.agal_dump(case._h, _lib.ARR_F, host_out.ctypes.data_as(C.c_void_p), host_out.nbytes)
    e2e_s = time.perf_counter() - t0
    if rc:
        raise RuntimeError("e2e run failed")
    e2e_s = allmax(e2e_s)
    case.close()
    e2e = {"value": allsum(float(e2e_cells)) / e2e_s / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": int(host_in.nbytes / a.steps),
           "d2h_bytes_per_step": int(host_out.nbytes / a.steps) + 8 * (dim + 1)}

    # --- roofline of the fused step kernel on a large case -------------------
    rwl = a.roofline_workload or ROOFLINE_FOR.get(w["storage"], "ldc2d_8192")
    rw = WORKLOADS[rwl]
    rcase = ag.Case(make_params(rw, device=local))
    rcase.set_ic(0)
    rtune = rcase.autotune(0, reps=5)
    for _ in range(3):
        rcase.advance()
    rcase.sync()
    rt, rcells, _ = time_steps(rcase, torch, rw, 20, flush=False)
    rcase.close()
    avg_ms = sum(rt) / len(rt)
    alg_bytes = 2 * Q_OF[rw["velocity_set"]] * ESIZE[rw["storage"]] * rcells[0]
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": dram_traffic_per_launch(rwl), "peak_source": peak_kind,
                "kernel": "k_step (fused collide+BC+stream) + its stream-guard fix-up",
                "workload": rwl, "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "autotune": rtune}

    # --- batched independent cases vs the same cases one at a time -----------
    batched = None
    if a.batched_cases > 0:
        batched = run_batched(torch, a.batched_cases, a.batched_seed, spinup=40, steps=20, device=local)

    # --- CPU baseline (rank 0 only) -------------------------------------------
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = run_cpu_oracle(w, seconds=a.cpu_seconds, threads=threads)

    if ws > 1:
        dist.destroy_process_group()
    if rank == 0:
        extra = {"parallelism": f"replicas x{ws}",
                 "l2": "flushed between timed steps" if head["flush"] else "inputs larger than L2",
                 "autotune": head["tune"], "blocks_per_level": head["counts"]["n_ids"][:-1],
                 "cell_updates_per_step": head["cells_per_step"]}
        line = dict(base, value=head["value"], ms_per_step=head["ms_per_step"],
                    config=config_of(a.workload, extra), e2e=e2e, roofline=roofline, cpu_baseline=cpu,
                    clocks=head["clocks"], gpu_launches=head["launches"])
        if plain is not None:
            line["plain_fp32"] = {"workload": a.plain_workload, "value": plain["value"],
                                  "ms_per_step": plain["ms_per_step"],
                                  "blocks_per_level": plain["counts"]["n_ids"][:-1],
                                  "ratio": head["value"] / plain["value"]}
        if learned is not None:
            mk = learned["plain_refine_marks"]
            learned["missed_fraction"] = learned["missed"] / mk if mk > 0 else 0.0
            if plain is not None:
                learned["ratio_vs_plain_fp32"] = learned["value"] / plain["value"]
            line["learned"] = learned
        if batched is not None:
            line["batched"] = batched
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
