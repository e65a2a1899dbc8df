#!/usr/bin/env python
"""Benchmark of the B200 octree-AMR lattice Boltzmann time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the headline configuration): D2Q9 lid-driven cavity on a 128^2
base grid in 4^2-cell blocks, up to 3 levels, refined above the 90th and
coarsened below the 50th percentile of the block vorticity every 64 coarse
steps, Re = 1000, lid 0.05, cubic interpolation, FP16 weight-offset
populations.  Seeded synthetic input: the fluid starts at rest and the
hierarchy develops in an untimed 1280-coarse-step spin-up.

One "step" is one regrid period: P_REFINE = 64 coarse steps
(Mesh::M_Advance_Step, the S_Advance recursion over every level) followed by
the solution-based refinement of the 64th (M_Advance_RefineWithSolution), so
every timed step holds exactly one regrid.  Metric: MLUPS, million lattice
cell updates per second, leaf cells of level L counted 2^L times per coarse
step as solver_lbm_advance.cu:74-89 counts them.

--impl b200 (default): the CUDA library.  Rank 0 prints one JSON line with
  value        device-timed MLUPS (CUDA events on the library's stream; the
               state is L2-resident, so L2 is flushed before every timed step)
  e2e          the same steps through the public C ABI with host buffers:
               the populations loaded from pinned host memory, K x (period +
               an asynchronous FP64 mass/momentum read back into pinned
               memory), the populations dumped; timed by wall clock
  plain_fp32   the same case in FP32 populations
  learned      the learned predictor on a 2D periodic vortex flow: trained on
               2000 snapshots labelled 4 regrids ahead, an FP16 run regridding
               4x less often (the rule judging every regrid) against plain
               FP16 / FP32 runs: MLUPS, regrid time per 1000 steps, missed
               refinements
  channel_d3q27  the D3Q27 icosphere channel (FP64 / FP32 / FP16 MLUPS and
               drag/lift against FP64)
  roofline     the fused step kernel on a large single-level case of the same
               physics (FP16 and FP32), algorithmic bytes 2*Q*s per update
  error_vs_fp64  rho and u of FP32 and FP16 runs of the headline case against
               an FP64 run of this library after --error-steps coarse steps
  cpu_baseline the CPU oracle (OpenMP restatement of the reference algorithm)
               on a bounded sample of the same workload, rank 0 only
--impl reference: the reference algorithm on the host cores (the CPU oracle
  port; the reference has no CPU implementation of its own), rank 0 only,
  plus the reference's own CUDA build (oracle/_ref) timed on this GPU where
  it was built.  Loads nothing of the agal_b200 native library.

Multi-GPU: one process per GPU under torchrun; every rank runs an
independent replica of the workload (a single case does not shard), so the
scaling is weak and `value` is the sum over ranks divided by the slowest
rank's time.  The batched measurement instead splits its fixed case list
across the ranks (LPT packing, agal_b200.shard): strong scaling, the sum of
the ranks' cell updates over the slowest rank's time.
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
    "amr_ldc2d_128_log2": dict(
        _AMR, storage=_lib.STORE_FP32, criterion=_lib.CRITERION_VORTICITY, refine_start=-2.0,
        desc="D2Q9 BGK lid-driven cavity, 128^2 base in 4^2-cell blocks, up to 3 levels, the reference's own "
             "criterion (floor(log2 |vorticity|) against N_REFINE_START -2, N_REFINE_INC 1, N_REFINE_MAX 1) every "
             "64 coarse steps, Re=1000, lid 0.05, cubic interpolation, FP32 populations"),
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


def make_params(w: dict, device: int = -1, defaults=None, **extra):
    """agal_params of a workload; `defaults` builds the parameter structure
    (the library's agal_params_default, or the oracle's restatement where the
    CUDA library must not be loaded)."""
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
        if w.get("criterion") is not None:
            kw.update(S_CRITERION=w["criterion"], N_REFINE_START=w["refine_start"], N_REFINE_INC=1.0,
                      N_REFINE_MAX=1.0)
    kw.update(extra)
    return (defaults or ag.default_params)(**kw)


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


FUSED_FIXUP_BLOCKS = 8192   # grids up to this many blocks apply the stream-guard fix-ups in their last CTA


def launches_per_step(counts: dict, amr: bool) -> int:
    """Kernels of one coarse step, from the structure of the level recursion:
    level L takes 2^L sub-steps, each a fused step (plus a separate
    stream-guard fix-up launch on grids of more than FUSED_FIXUP_BLOCKS
    blocks), and every non-empty level below the finest launches 2^L
    interpolations and 2^L averagings; the rounding counter's tick rides on
    the last averaging."""
    if not amr:
        return 2
    n, ml = counts["n_ids"], counts["max_levels"]
    total = 0
    for L in range(ml):
        if n[L] == 0:
            continue
        mult = 1 << L
        total += mult * (2 if n[L] > FUSED_FIXUP_BLOCKS else 1)
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
def coarse_per_step(w: dict) -> int:
    """Coarse steps in one bench step: a whole regrid period for multi-level
    workloads, one for single-level ones."""
    return w["p_refine"] if w.get("amr") else 1


def step_fn(case, w: dict):
    """One bench step: a captured regrid period (its 64th coarse step ends
    with the refinement) or one fused single-level step."""
    if w.get("amr"):
        n = coarse_per_step(w)
        return lambda: case.advance_n(n, use_graph=True)
    return case.advance


def time_steps(case, torch, w: dict, n_steps: int, flush: bool):
    """Per-step device time (ms) with CUDA events on the library's stream,
    the cell updates and the library kernel launches of each step."""
    stream = torch.cuda.ExternalStream(case.stream_ptr())
    scratch = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda") if flush else None
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
    step = step_fn(case, w)
    dim = DIM_OF[w["velocity_set"]]
    k = coarse_per_step(w)
    cells, launches = [], 0
    for i in range(n_steps):
        if flush:
            with torch.cuda.stream(stream):
                scratch.add_(1.0)   # writes 252 MB > L2 between timed steps
        cnt = case.counts()   # the mesh holds for the whole period (regrid at its end)
        cells.append(k * leaf_cells(cnt, dim))
        launches += k * launches_per_step(cnt, w.get("amr", False))
        if w.get("amr"):
            launches += regrid_launches(cnt)
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    case.sync()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs], cells, launches


def develop(case, w: dict):
    """Initial state, then the untimed spin-up that builds the hierarchy (a
    whole number of regrid periods, so that bench steps start on a period)."""
    case.set_ic(0)
    if w.get("amr"):
        case.refine_near_wall()
        case.advance_n(w["spinup"], use_graph=True)
        assert case.refine_stats()["iter"] % w["p_refine"] == 0


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


def run_batched(torch, n_cases: int, seed: int, spinup: int, steps: int, device: int,
                rank: int = 0, ws: int = 1, allsum=None, allmax=None, barrier=None) -> dict:
    """Aggregate MLUPS of the batch (FP16 populations, batched graph) and of
    the same cases in FP32 advanced one at a time; both after the same
    spin-up, timed with CUDA events over `steps` coarse steps that hold no
    regrid (P_REFINE = 32, spin-up past the first regrid).  Under torchrun the
    case list is split across the ranks by LPT packing (agal_b200.shard): each
    rank builds and times only its cases; the figures are the sum of the
    ranks' cell updates over the slowest rank's time."""
    from agal_b200.shard import aggregate, case_cost, lpt_shards, shard_loads
    allsum = allsum or (lambda x: x)
    allmax = allmax or (lambda x: x)
    barrier = barrier or (lambda: None)
    specs_all = batched_specs(n_cases, seed)
    costs = [case_cost(s) for s in specs_all]
    shards = lpt_shards(costs, ws)
    specs = [specs_all[i] for i in shards[rank]]

    def build(storage):
        cases = [batched_case(s, storage, device) for s in specs]
        tunes = [c.autotune(0, reps=3)["variant"] for c in cases]
        return cases, tunes

    def cells(cases):
        return sum(leaf_cells(c.counts(), 3) for c in cases)

    # batched, FP16: the autotuner picks the launch mode (work list or one
    # graph branch per case); both modes are then timed over 20 coarse steps
    # that hold no regrid (P_REFINE = 32)
    cases, tunes16 = build(_lib.STORE_FP16)
    batch = ag.Batch(cases)
    batch.advance_n(spinup)
    tuned = batch.autotune(4)
    at = spinup + 2 * (4 + 2)
    stream = torch.cuda.ExternalStream(batch.stream())

    def timed_window(start_at):
        """Advance to step `start_at`, then time `steps` coarse steps."""
        batch.advance_n(start_at - timed_window.at)
        batch.sync()
        upd = cells(cases)
        barrier()
        a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_.record(stream)
        batch.advance_n(steps)
        b_.record(stream)
        batch.sync()
        timed_window.at = start_at + steps
        return upd, a_.elapsed_time(b_)
    timed_window.at = at
    period = 32
    first = (at + period - 1) // period * period          # the step after a regrid
    upd16, t16 = timed_window(first)
    levels16 = [c.counts()["n_ids"][:-1] for c in cases]
    # the other mode, in the next regrid-free window
    batch.set_worklist(not tuned["worklist"])
    upd16b, t16b = timed_window((timed_window.at + period - 1) // period * period)
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
    agg16b = aggregate(upd16b * steps, t16b, allsum, allmax)
    agg16 = aggregate(upd16 * steps, t16, allsum, allmax)
    agg32 = aggregate(upd32 * steps, t32, allsum, allmax)
    v16, v32 = agg16["mlups"], agg32["mlups"]
    upd16, upd32 = agg16["cell_updates"] / steps, agg32["cell_updates"] / steps
    t16, t32 = agg16["ms"], agg32["ms"]
    peak, kind = measured_peak_hbm()
    gbs = upd16 * steps * 2 * 19 * 2 / (t16 * 1e-3) / 1e9 / ws   # per GPU
    return {"workload": "batched_d3q19_64", "n_cases": n_cases, "seed": seed,
            "desc": "independent D3Q19 BGK cases, base N^3 with N in {32,48,64,96}, 1-3 levels, Re log-uniform "
                    "[100,1000], half lid-driven cavities with percentile solution refinement, half flow past "
                    "a seeded ellipsoid (axes 8-24 cells) with near-wall refinement, interpolated bounce-back "
                    "and MEA forces; refinement by the plain criterion (no learned predictor)",
            "spinup_steps": spinup, "timed_steps": steps,
            "sharding": {"ranks": ws, "scaling": "strong" if ws > 1 else "n/a",
                         "packing": "LPT on base cells x 2^(levels-1)",
                         "cases_per_rank": [len(x) for x in shards],
                         "load_per_rank": shard_loads(costs, shards)},
            "value": v16, "unit": "MLUPS", "storage": "f16-offset", "ms_per_step": t16 / steps,
            "cell_updates_per_step": upd16,
            "one_at_a_time_fp32": {"value": v32, "ms_per_step": t32 / steps, "cell_updates_per_step": upd32},
            "other_mode_fp16": {"value": agg16b["mlups"], "ms_per_step": agg16b["ms"] / steps,
                                "mode": "graph branches" if tuned["worklist"] else "work list"},
            "mode": "work list" if tuned["worklist"] else "graph branches",
            "autotune": tuned,
            "modes": "work list: one persistent step kernel per phase over all cases' (case, chunk) items, batched "
                     "fix-ups, one launch per interpolation / averaging phase over (case, parent block) items, walls "
                     "and forces per case; graph branches: each case's launches as its own branch of the graph",
            "ratio_vs_one_at_a_time_fp32": v16 / v32,
            "hbm": {"achieved_gbs_per_gpu": gbs, "peak": peak, "frac": gbs / peak, "peak_source": kind,
                    "bytes_per_update": 2 * 19 * 2},
            "autotune_variants": {"fp16": tunes16, "fp32": tunes32},
            "blocks_per_level_fp16": levels16, "blocks_per_level_of": "rank 0's cases"}


def run_cpu_oracle(w: dict, seconds: float, threads: int, max_steps: int | None = None) -> dict:
    """Oracle (CPU restatement, OpenMP) MLUPS on a bounded sample of the
    workload, after the same spin-up; parameters from the oracle's own
    defaults, so no native code of agal_b200 is loaded here."""
    from oracle.orc import OracleCase, build, default_params  # CPU baseline / reference arm only
    build()
    p = make_params(w, defaults=default_params)
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


def reference_cuda(timeout_s: float = 600.0) -> dict:
    """The reference's own CUDA build (oracle/_ref, compiled from its sources by
    `make -C oracle ref`) timed on this GPU with CUDA events around its
    M_Advance_Step loop (oracle/ref_harness/ref_main.cu; the reference
    synchronises after every kernel, solver_lbm_advance.cu:72-89): the
    single-level 256^2 cavity (Re 100) and the 3-level 128^2 cavity with its own
    log2 vorticity criterion (Re 1000, regrid every 64 steps, 1280-step
    spin-up; the timed steps hold no regrid, as the harness times them)."""
    from oracle.ref_run import REF_BIN, run_ref   # reference arm only
    out = {"source": "oracle/_ref/ref_d2q9_ldc (the reference's sources, nvcc sm_100a)"}
    if not (REF_BIN / "ref_d2q9_ldc").exists():
        out["unavailable"] = "oracle/_ref/ref_d2q9_ldc was not built (no reference tree where build() ran)"
        return out
    w2 = WORKLOADS["amr_ldc2d_128_log2"]
    runs = {
        "ldc2d_256": (dict(Nx=256, v0=5e-4), 3, 2000),
        "amr_ldc2d_128_log2": (dict(Nx=128, v0=0.05 / w2["Re"], MAX_LEVELS_INTERIOR=w2["levels"],
                                    P_REFINE=w2["p_refine"], S_CRITERION=0, N_REFINE_START=w2["refine_start"],
                                    N_REFINE_INC=1.0, N_REFINE_MAX=1.0), w2["spinup"], 1280),
    }
    for name, (keys, spin, timed) in runs.items():
        try:
            txt = run_ref("ref_d2q9_ldc", keys, spin, 4096, None, n_timed=timed)
            line = [ln for ln in txt.splitlines() if ln.startswith('{"ref_timing"')]
            out[name] = json.loads(line[-1]) if line else {"error": txt[-300:]}
        except Exception as e:   # noqa: BLE001 - reported, not fatal
            out[name] = {"error": str(e)[-300:]}
    return out


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


def _copy_state(src, dst):
    """Every mesh array, the populations and the counts of src into dst."""
    for arr in (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_F_X, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR,
                _lib.ARR_CBLOCK_ID_NBR_CHILD, _lib.ARR_CBLOCK_ID_ONB, _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL,
                _lib.ARR_ID_SET, _lib.ARR_GAP_SET, _lib.ARR_F):
        dst.load(arr, src.dump(arr))
    cnt = src.counts()
    dst.set_counts(cnt["n_ids"], cnt["id_max"], cnt["n_gaps"])


def _rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def error_vs_fp64(wl: str, steps: int, device: int) -> dict:
    """Precision of FP32 and FP16 storage against FP64 runs of this library
    on the headline case, after `steps` coarse steps:
      same_mesh    every storage continues the FP64 run's state after its
                   spin-up, without regrids (the storage error alone), rho and
                   u of every active cell;
      independent  each storage runs the whole case with its own regrids (the
                   meshes may differ: fields compared on the uniform grid of
                   the finest level, prepared as the reference's
                   M_Advance_PrintData prepares its output);
      drag, lift   momentum-exchange forces of a tilted ellipsoid (D3Q19 64^3,
                   two near-wall levels, interpolated bounce-back, Re 100,
                   3,000 steps)."""
    ww = dict(WORKLOADS[wl])
    dim, Q = DIM_OF[ww["velocity_set"]], Q_OF[ww["velocity_set"]]
    pb = {9: [0, 3, 4, 1, 2, 7, 8, 5, 6]}[Q]

    def leaf(c, p):
        nmb, MC = p.n_maxcblocks, 4 ** dim
        cnt = c.counts()
        ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
        blocks = np.sort(np.concatenate([ids[L, :cnt["n_ids"][L]] for L in range(cnt["max_levels"])]))
        F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks.astype(np.int64), :].reshape(Q, -1)
        cx = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])[pb]   # slot s holds f_{pb(s)}
        cy = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])[pb]
        rho = F.sum(axis=0)
        return rho, np.stack([(cx[:, None] * F).sum(axis=0) / rho, (cy[:, None] * F).sum(axis=0) / rho])

    out = {"workload": wl, "coarse_steps": steps, "bar_u_rel_l2": 1e-3}
    same, indep = {}, {}
    p64 = make_params(dict(ww, storage=_lib.STORE_FP64), device=device)
    with ag.Case(p64) as s:
        s.set_ic(0)
        s.refine_near_wall()
        s.advance_n(ww["spinup"], use_graph=True)
        s.sync()
        for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
            p = make_params(dict(ww, storage=st), device=device, P_REFINE=10 ** 8)
            with ag.Case(p) as c:
                _copy_state(s, c)
                c.advance_n(steps - ww["spinup"], use_graph=True)
                c.sync()
                same[name] = leaf(c, p)
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
        w = dict(ww, storage=st)
        p = make_params(w, device=device, N_PRINT_LEVELS=w["levels"], VOL_I_MIN=0, VOL_I_MAX=w["Nx"],
                        VOL_J_MIN=0, VOL_J_MAX=w["Nx"])
        with ag.Case(p) as c:
            c.set_ic(0)
            c.refine_near_wall()
            c.advance_n(steps, use_graph=True)
            c.sync()
            indep[name] = (c.render_prepared(), c.counts()["n_ids"][: w["levels"]])
    forces = drag_lift(device)
    for name in ("fp32", "fp16"):
        f, blocks = indep[name]
        r0 = indep["fp64"][0]
        out[name] = {"same_mesh": {"rho_rel_l2": _rel(same[name][0], same["fp64"][0]),
                                   "u_rel_l2": _rel(same[name][1], same["fp64"][1])},
                     "independent": {"rho_rel_l2": _rel(f["rho"], r0["rho"]),
                                     "u_rel_l2": _rel(np.stack([f["u"], f["v"]]), np.stack([r0["u"], r0["v"]])),
                                     "blocks_per_level": blocks},
                     "drag_rel": abs(forces[name][0] - forces["fp64"][0]) / abs(forces["fp64"][0]),
                     "lift_rel": abs(forces[name][1] - forces["fp64"][1]) / abs(forces["fp64"][1])}
    out["independent_blocks_per_level_fp64"] = indep["fp64"][1]
    out["drag_lift_case"] = ("tilted ellipsoid (semi-axes 0.16, 0.07, 0.08 of the unit box, 20 degrees about z), "
                             "D3Q19 64^3, two near-wall levels, interpolated bounce-back, second-order momentum "
                             "exchange, inflow 0.05, Re 100, forces of step 3,000")
    out["fp64_drag_lift"] = [float(forces["fp64"][0]), float(forces["fp64"][1])]
    return out


def drag_lift(device: int) -> dict:
    from agal_b200.geometry import icosphere
    f = icosphere(3, 1.0, (0, 0, 0), seed=9).astype(np.float64)
    th = 0.35
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    f = ((f * np.array([0.16, 0.07, 0.08])) @ R.T + np.array([0.42, 0.5, 0.5])).astype(np.float32)
    out = {}
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
        p = ag.default_params(velocity_set=_lib.D3Q19, Nx=64, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1,
                              v0=0.05 * 0.32 / 100, P_REFINE=10 ** 8, G_BIN_DENSITY=8, G_BIN_LEVELS=2, G_BIN_SPEC=2,
                              G_BIN_MAKE_LINKS=1, G_NEAR_WALL_DISTANCE=0.05, S_BC_TYPE=1, S_FORCE_TYPE=0,
                              S_FORCE_ORDER=2, bc_preset=_lib.BC_FPSC3D, ic_preset=_lib.IC_UNIFORM, u_ref=0.05,
                              storage=st, n_maxcblocks=4096 * 4 + 64, device=device)
        with ag.Case(p) as c:
            c.set_geometry(f)
            c.set_ic(0)
            c.refine_near_wall()
            c.advance_n(2999, use_graph=True)
            c.forces()
            c.advance_n(1, use_graph=True)
            fr = c.forces()
            out[name] = np.array([fr[0] - fr[1], fr[2] - fr[3], fr[4] - fr[5]])
    return out


def _vortex_params(storage: int, p_refine: int, device: int, seed: int = 2024):
    """2D periodic flow carrying vortices across the domain: D2Q9 128^2,
    periodic in x and y, uniform u = 0.05 with 30% seeded velocity noise,
    Re 500, up to 3 levels by the percentile rule (refine > p90, coarsen <
    p50) every `p_refine` coarse steps, cubic interpolation."""
    nb = 32 * 32
    return ag.default_params(velocity_set=_lib.D2Q9, Nx=128, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=3,
                             P_REFINE=p_refine, S_CRITERION=_lib.CRITERION_PERCENTILE, ref_pct_hi=0.9,
                             ref_pct_lo=0.5, interp_order=_lib.INTERP_CUBIC, PERIODIC_X=1, PERIODIC_Y=1,
                             bc_preset=_lib.BC_NONE, ic_preset=_lib.IC_UNIFORM, u_ref=0.05, ic_noise=0.3,
                             seed=seed, v0=0.05 / 500.0, storage=storage, n_maxcblocks=nb * 21 + 64,
                             device=device)


def _time_periods(torch, case, period: int, n_periods: int) -> dict:
    """Device time of n_periods regrid periods, split into the coarse steps
    and the regrid (the last coarse step's time beyond a plain step's)."""
    stream = torch.cuda.ExternalStream(case.stream_ptr())
    total = regrid = 0.0
    cells = 0
    for _ in range(n_periods):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        cells += period * leaf_cells(case.counts(), 2)
        e0.record(stream)
        case.advance_n(period - 1, use_graph=True)
        e1.record(stream)
        case.advance_n(1, use_graph=True)   # the last step and its regrid
        e2.record(stream)
        case.sync()
        t_steps, t_last = e0.elapsed_time(e1), e1.elapsed_time(e2)
        total += t_steps + t_last
        regrid += max(t_last - t_steps / (period - 1), 0.0)
    steps = period * n_periods
    return {"mlups": cells / (total * 1e-3) / 1e6, "ms": total, "coarse_steps": steps,
            "regrids": n_periods, "regrids_per_1000_steps": 1000.0 * n_periods / steps,
            "regrid_ms_per_1000_steps": 1000.0 * regrid / steps, "blocks_per_level": case.counts()["n_ids"][:-1]}


def _batched_vortices(torch, device: int, weights, thr, horizon: int, base: int, n_cases: int = 8,
                      spinup: int = 512, window: int = 512) -> dict:
    """The learned predictor inside a batch: n_cases periodic-vortex cases
    (other noise seeds) advanced together (one graph branch per case), FP16,
    once with the percentile rule every `base` coarse steps and once each
    driven by its own copy of the trained network every base x horizon steps
    (the rule judging every regrid).  MLUPS over `window` coarse steps after
    `spinup`, device time on the batch stream, regrids included."""
    out = {"n_cases": n_cases, "spinup_steps": spinup, "window_steps": window}
    for name, period, learned in (("plain_fp16", base, False), ("learned_fp16", base * horizon, True)):
        cases, nets = [], []
        for i in range(n_cases):
            c = ag.Case(_vortex_params(_lib.STORE_FP16, period, device, seed=3000 + i))
            if learned:
                n = ag.Learner(2, seed=7)
                n.set_params(weights)
                n.set_horizon(horizon)
                n.attach(c, 2, judge_every=1)
                n.set_thresholds(*thr)
                nets.append(n)
            c.set_ic(0)
            c.refine_near_wall()
            cases.append(c)
        with ag.Batch(cases) as b:
            b.set_worklist(False)
            b.advance_n(spinup)
            b.sync()
            stream = torch.cuda.ExternalStream(b.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            cells = 0
            e0.record(stream)
            for _ in range(window // base):
                cells += base * sum(leaf_cells(c.counts(), 2) for c in cases)
                b.advance_n(base)
            e1.record(stream)
            b.sync()
            ms = e0.elapsed_time(e1)
        out[name] = {"mlups": cells / (ms * 1e-3) / 1e6, "ms": ms, "regrids_per_case": window // period}
        for n in nets:
            n.close()
        for c in cases:
            c.close()
    out["ratio_learned_vs_plain"] = out["learned_fp16"]["mlups"] / out["plain_fp16"]["mlups"]
    return out


def learned_ahead(torch, device: int, horizon: int = 4, n_snap: int = 2000, epochs: int = 2,
                  window: int = 1024, spinup: int = 1024) -> dict:
    """The learned predictor adapting the grid less often, on the periodic
    vortex flow (_vortex_params).  The network is trained on n_snap snapshots
    of the plain FP32 run (a regrid every 16 coarse steps), each labelled with
    the percentile rule's decisions over the next `horizon` regrids; a fresh
    FP16 run driven by the network regrids every horizon x 16 steps, the rule
    judging every regrid (its refinements the network missed are counted and
    applied).  Against the plain FP16 and FP32 runs regridding every 16 steps,
    after the same spin-up: MLUPS, device time, regrids and regrid time per
    1000 coarse steps, and the missed-refinement fraction (the meshes differ, so
    MLUPS counts different cells: the device time of the same coarse steps is
    the like-for-like figure); then the same comparison for 8 such cases
    advanced as one batch (`batched`)."""
    base = 16
    t0 = time.perf_counter()
    src = ag.Case(_vortex_params(_lib.STORE_FP32, base, device))
    m = ag.Learner(2, seed=7)
    m.set_horizon(horizon)
    m.attach(src, 1)
    src.set_ic(0)
    src.refine_near_wall()
    src.advance_n(base * (n_snap + horizon), use_graph=True)
    src.sync()
    collect_s = time.perf_counter() - t0
    nl = m.counts()["labelled"]
    weights = m.balance_classes(0, nl)
    loss = m.train(0, nl, epochs, lr=2e-3, seed=7)
    thr = m.calibrate_thresholds(0, nl)
    m.attach(src, 0)
    src.close()
    train_s = time.perf_counter() - t0 - collect_s
    out = {"workload": "vortices2d_128_periodic", "desc": _vortex_params.__doc__.split("\n\n")[0].strip(),
           "horizon": horizon, "snapshots": nl, "epochs": epochs, "class_weights": weights, "train_loss": loss,
           "thresholds": thr, "collect_s": collect_s, "train_s": train_s, "spinup_steps": spinup}
    runs = (("plain_fp32", _lib.STORE_FP32, base, False), ("plain_fp16", _lib.STORE_FP16, base, False),
            ("learned_fp16", _lib.STORE_FP16, base * horizon, True))
    meshes = {}

    def refined_cells(c):
        """Root-grid positions covered by each finer level (2D), as sets."""
        cnt = c.counts()
        nmb = c.params.n_maxcblocks
        ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
        fx = c.dump(_lib.ARR_CBLOCK_F_X).reshape(2, nmb)
        out = {}
        for L in range(1, cnt["max_levels"]):
            b = ids[L, : cnt["n_ids"][L]].astype(np.int64)
            out[L] = {(int(round(x * 128 * 2 ** L)), int(round(y * 128 * 2 ** L))) for x, y in zip(fx[0, b], fx[1, b])}
        return out

    for name, st, period, learned in runs:
        c = ag.Case(_vortex_params(st, period, device))
        if learned:
            m.attach(c, 2, judge_every=1)
            m.set_thresholds(*thr)
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(spinup, use_graph=True)
        c.autotune(0, reps=5)
        c0 = m.counts()
        r = _time_periods(torch, c, period, window // period)
        if learned:
            c1 = m.counts()
            r.update(judged=c1["judged"] - c0["judged"], plain_refine_marks=c1["plain_refine"] - c0["plain_refine"],
                     missed=c1["missed"] - c0["missed"])
            r["missed_fraction"] = r["missed"] / r["plain_refine_marks"] if r["plain_refine_marks"] else 0.0
            m.attach(c, 0)
        meshes[name] = refined_cells(c)
        c.close()
        out[name] = r
    out["batched"] = _batched_vortices(torch, device, m.get_params(), thr, horizon, base)
    m.close()
    # both runs end on a regrid of theirs at the same coarse step: the share of
    # the plain FP16 run's refined blocks (per level) the learned run also has
    def coverage(ref, other):
        return {f"L{L}": (len(pl & meshes[other].get(L, set())) / len(pl) if pl else 1.0)
                for L, pl in meshes[ref].items()}
    out["learned_fp16"]["coverage_of_plain_mesh"] = coverage("plain_fp16", "learned_fp16")
    # the same measure between the two plain runs (FP32 against FP16): how far
    # two runs of this flow drift apart in where they refine
    out["plain_fp32"]["coverage_of_plain_fp16_mesh"] = coverage("plain_fp16", "plain_fp32")
    out["regrid_ms_saved_per_1000_steps"] = (out["plain_fp16"]["regrid_ms_per_1000_steps"] -
                                             out["learned_fp16"]["regrid_ms_per_1000_steps"])
    out["ratio_learned_fp16_vs_plain_fp32"] = out["learned_fp16"]["mlups"] / out["plain_fp32"]["mlups"]
    out["ratio_learned_fp16_vs_plain_fp16"] = out["learned_fp16"]["mlups"] / out["plain_fp16"]["mlups"]
    return out


def config4(torch, device: int, steps: int) -> dict:
    """The D3Q27 icosphere channel: external flow over a seeded icosphere
    (20,480 faces, diameter 32 root cells) in a 256 x 128 x 128 channel, 4
    levels with the finest band around the body (near-wall refinement),
    uniform inflow u = 0.05 with seeded 1% noise, Re = 200 on the diameter,
    interpolated bounce-back and momentum-exchange forces.  FP64, FP32 and
    FP16 storage run the same `steps` coarse steps; drag and lift are the MEA
    forces of the last one; MLUPS over 20 coarse steps (CUDA events).  The
    reference's own build cannot run this box like for like (its bins assume
    the unit cube), so FP64 of this library is the judge."""
    from agal_b200.geometry import icosphere
    N, R = 256, 16.0 / 256
    faces = icosphere(5, R, (0.25, 0.25, 0.25), seed=2024)
    out = {"workload": "channel3d27_256x128x128_icosphere", "n_faces": int(len(faces)), "coarse_steps": steps,
           "desc": "D3Q27 BGK channel 256x128x128 (1 x 0.5 x 0.5), seeded icosphere of 20,480 faces, diameter 32 "
                   "root cells, 4 levels near the wall, inflow 0.05 with 1% seeded noise, Re 200, Bouzidi walls, "
                   "MEA drag/lift; plain criterion only"}
    forces = {}
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
        p = ag.default_params(velocity_set=_lib.D3Q27, Nx=N, L_fy=0.5, L_fz=0.5, MAX_LEVELS_WALL=4,
                              MAX_LEVELS_INTERIOR=1, v0=0.05 * 2 * R / 200.0, P_REFINE=10 ** 8, G_BIN_DENSITY=8,
                              G_BIN_LEVELS=4, G_BIN_SPEC=2, G_BIN_MAKE_LINKS=1, G_NEAR_WALL_DISTANCE=0.02,
                              S_BC_TYPE=1, S_FORCE_TYPE=0, S_FORCE_ORDER=2, bc_preset=_lib.BC_FPSC3D,
                              ic_preset=_lib.IC_UNIFORM, u_ref=0.05, ic_noise=0.01, seed=2024,
                              interp_order=_lib.INTERP_LINEAR, storage=st, n_maxcblocks=500000, device=device)
        with ag.Case(p) as c:
            c.set_geometry(faces)
            c.set_ic(0)
            c.refine_near_wall()
            c.autotune(0, reps=3)
            n_pre = max(steps - 21, 0)
            c.advance_n(n_pre, use_graph=True)
            cnt = c.counts()
            upd = leaf_cells(cnt, 3)
            c.sync()
            stream = torch.cuda.ExternalStream(c.stream_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c.advance_n(20, use_graph=True)
            e1.record(stream)
            c.sync()
            ms = e0.elapsed_time(e1) / 20
            c.forces()                       # partials reset: the last step's forces follow
            c.advance_n(steps - n_pre - 20, use_graph=True)
            fr = c.forces()
            forces[name] = np.array([fr[0] - fr[1], fr[2] - fr[3], fr[4] - fr[5]])
            out[name] = {"mlups": upd / (ms * 1e-3) / 1e6, "ms_per_coarse_step": ms, "cell_updates_per_step": upd,
                         "blocks_per_level": cnt["n_ids"][:-1], "drag": float(forces[name][0]),
                         "lift": [float(forces[name][1]), float(forces[name][2])]}
    ref = forces["fp64"]
    for name in ("fp32", "fp16"):
        out[name]["drag_rel_vs_fp64"] = float(abs(forces[name][0] - ref[0]) / abs(ref[0]))
        out[name]["lift_rel_vs_fp64_drag"] = float(np.abs(forces[name][1:] - ref[1:]).max() / abs(ref[0]))
    out["fp16_over_fp32_mlups"] = out["fp16"]["mlups"] / out["fp32"]["mlups"]
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30, help="timed steps (regrid periods of the AMR workload)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="amr_ldc2d_128_fp16", choices=sorted(WORKLOADS))
    ap.add_argument("--plain-workload", default="amr_ldc2d_128", choices=sorted(WORKLOADS),
                    help="the same case in plain FP32, timed beside the headline workload")
    ap.add_argument("--roofline-workload", default=None, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--learn-snapshots", type=int, default=2000,
                    help="snapshots the learned predictor is trained on (0 skips the learned leg)")
    ap.add_argument("--learn-horizon", type=int, default=4, help="regrid periods the predictor looks ahead")
    ap.add_argument("--learn-epochs", type=int, default=2)
    ap.add_argument("--config4-steps", type=int, default=600,
                    help="coarse steps of the D3Q27 icosphere channel leg (0 skips it)")
    ap.add_argument("--error-steps", type=int, default=20000,
                    help="coarse steps of the FP32/FP16-vs-FP64 error runs (0 skips them)")
    ap.add_argument("--profile", choices=sorted(WORKLOADS), default=None,
                    help="only run W+K steps of this workload (for ncu captures); prints no JSON line")
    ap.add_argument("--cpt", type=int, default=1, choices=[1, 2, 3, 4, 5, 6],
                    help="with --profile: step kernel variant (1, 2 cells per thread; 3 TMA pipeline; "
                         "4 one row of four cells per thread; 5 root-level tiles, 2D)")
    ap.add_argument("--batched-cases", type=int, default=64,
                    help="independent D3Q19 cases of the batched measurement (0 skips it)")
    ap.add_argument("--batched-seed", type=int, default=2024)
    ap.add_argument("--spinup", type=int, default=None,
                    help="with --profile: coarse steps of the untimed spin-up of a multi-level workload")
    ap.add_argument("--profile-batched", action="store_true",
                    help="only build the batched cases (FP16), advance 40 coarse steps, then 2 inside "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off); prints no JSON line")
    a = ap.parse_args(argv)
    a.warmup = max(a.warmup, 3)
    w = WORKLOADS[a.workload]
    if a.profile_batched:
        import torch
        specs = batched_specs(a.batched_cases, a.batched_seed)
        cases = [batched_case(sp, _lib.STORE_FP16, 0) for sp in specs]
        for c in cases:
            c.autotune(0, reps=3)
        with ag.Batch(cases) as b:
            b.advance_n(40)
            b.sync()
            torch.cuda.cudart().cudaProfilerStart()
            b.advance_n(2)
            b.sync()
            torch.cuda.cudart().cudaProfilerStop()
        for c in cases:
            c.close()
        print(f"batched profile run done: {len(cases)} cases, 40 + 2 coarse steps")
        return 0
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
    per = coarse_per_step(w)
    base = {"metric": "MLUPS (lattice cell updates per second / 1e6); one step = one regrid period of "
                      f"{per} coarse time steps including its refinement",
            "unit": "MLUPS", "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE_NAME[w["storage"]], "data": "synthetic (fluid at rest, lid-driven)"}

    def config_of(wl: str, extra: dict) -> dict:
        ww = WORKLOADS[wl]
        cfg = {"workload": wl, "desc": ww["desc"]}
        if ww.get("amr"):
            cfg.update(base_grid=f"{ww['Nx']}^2", levels=ww["levels"], regrid_every=ww["p_refine"],
                       coarse_steps_per_step=coarse_per_step(ww), spinup_steps=ww["spinup"])
        cfg.update(extra)
        return cfg

    if a.impl == "reference":
        # The reference algorithm on the host cores, plus the reference's own
        # CUDA build; other ranks idle.  Nothing of agal_b200's native code.
        if rank != 0:
            return 0
        steps = a.steps * per
        cb = run_cpu_oracle(w, seconds=1e9, threads=threads, max_steps=steps)
        line = dict(base, impl="reference", value=cb["value"], ms_per_step=None,
                    config=config_of(a.workload, {"parallelism": "host OpenMP", "l2": "n/a (CPU)"}),
                    cpu_baseline=cb, e2e={"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0})
        line["n_gpus"] = 0
        line["reference_cuda"] = reference_cuda()
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

    def device_timed(wl: str, with_clocks: bool, steps: int):
        ww = WORKLOADS[wl]
        case = ag.Case(make_params(ww, device=local))
        develop(case, ww)
        tune = case.autotune(0, reps=10)
        step = step_fn(case, ww)
        flush = state_bytes(case, ww) * 2 < L2_BYTES
        clk = ClockSampler(local) if with_clocks else None
        if clk:
            clk.__enter__()
            time.sleep(1.0)   # nvidia-smi is sampling before the warm-up starts
        for _ in range(a.warmup):
            step()
        case.sync()
        barrier()
        torch.cuda.synchronize()
        it0 = case.refine_stats()
        per_step, cells, launches = time_steps(case, torch, ww, steps, flush)
        it1 = case.refine_stats()
        clocks = None
        if clk:
            clk.__exit__(None, None, None)
            clocks = clk.summary()
        counts = case.counts()
        barrier()
        t_ms = allmax(sum(per_step))
        mlups = allsum(float(sum(cells))) / (t_ms * 1e-3) / 1e6
        case.close()
        regrids = (it1["iter"] - it0["iter"]) // ww["p_refine"] if ww.get("amr") else 0
        return dict(value=mlups, ms_per_step=t_ms / steps, flush=flush, tune=tune, clocks=clocks,
                    launches=launches, counts=counts, cells_per_step=float(np.mean(cells)), regrids=regrids,
                    ms_per_coarse_step=t_ms / steps / coarse_per_step(ww))

    def e2e_timed(wl: str, variant: int, steps: int) -> dict:
        """The same steps through the public C ABI with host buffers."""
        ww = WORKLOADS[wl]
        case = ag.Case(make_params(ww, device=local))
        develop(case, ww)
        case.set_tuning(variant)
        f0 = case.dump(_lib.ARR_F)
        host_in = torch.from_numpy(f0).pin_memory().numpy()
        host_out = torch.empty(f0.shape, dtype=torch.float64).pin_memory().numpy()
        mm = torch.zeros((steps, 4), dtype=torch.float64).pin_memory().numpy()
        lib = _lib.lib()
        dim = DIM_OF[ww["velocity_set"]]
        k = coarse_per_step(ww)
        amr = bool(ww.get("amr"))
        cells = 0
        barrier()
        t0 = time.perf_counter()
        rc = lib.agal_load(case._h, _lib.ARR_F, host_in.ctypes.data_as(C.c_void_p), host_in.nbytes)
        for i in range(steps):
            cells += k * leaf_cells(case.counts(), dim)
            rc |= lib.agal_advance_n(case._h, k, 1) if amr else lib.agal_advance(case._h, 0)
            rc |= lib.agal_mass_momentum_async(case._h, mm[i].ctypes.data_as(C.c_void_p))
        rc |= lib.agal_dump(case._h, _lib.ARR_F, host_out.ctypes.data_as(C.c_void_p), host_out.nbytes)
        rc |= lib.agal_sync(case._h)
        dt = time.perf_counter() - t0
        if rc:
            raise RuntimeError("e2e run failed: " + case._lib.agal_last_error(case._h).decode())
        dt = allmax(dt)
        case.close()
        drift = float(np.abs(mm[:, 0] - mm[0, 0]).max() / mm[0, 0])
        return {"value": allsum(float(cells)) / dt / 1e6, "unit": "MLUPS",
                "h2d_bytes_per_step": int(host_in.nbytes / steps),
                "d2h_bytes_per_step": int(host_out.nbytes / steps) + 8 * 4,
                "wall_ms_per_step": dt * 1e3 / steps, "mass_rel_drift": drift}

    def roofline_of(rwl: str) -> dict:
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
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": dram_traffic_per_launch(rwl), "peak_source": peak_kind,
                "kernel": "fused collide+BC+stream step (autotuned variant) + its stream-guard fix-up",
                "workload": rwl, "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "autotune": rtune}

    # --- device-timed steps: headline workload, learned, plain FP32 --------
    head = device_timed(a.workload, with_clocks=True, steps=a.steps)
    learned = learned_ahead(torch, local, horizon=a.learn_horizon, n_snap=a.learn_snapshots,
                            epochs=a.learn_epochs) if a.learn_snapshots > 0 else None
    plain = device_timed(a.plain_workload, with_clocks=False, steps=a.steps) \
        if a.plain_workload != a.workload else None
    # the reference's own criterion, timed like the reference harness times
    # it (coarse steps after the spin-up, no regrid in the window)
    ref_rule = None
    if w.get("amr"):
        wr = WORKLOADS["amr_ldc2d_128_log2"]
        c = ag.Case(make_params(wr, device=local))
        develop(c, wr)
        c.autotune(0, reps=5)
        c.sync()
        st = torch.cuda.ExternalStream(c.stream_ptr())
        cells, ms_tot, n_t = 0, 0.0, 0
        for _ in range(20):
            # the first 63 coarse steps of a period (no refinement turn) timed,
            # then the 64th with its regrid untimed
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            cells += (wr["p_refine"] - 1) * leaf_cells(c.counts(), 2)
            e0.record(st)
            c.advance_n(wr["p_refine"] - 1, use_graph=True)
            e1.record(st)
            c.advance_n(1, use_graph=True)
            c.sync()
            ms_tot += e0.elapsed_time(e1)
            n_t += wr["p_refine"] - 1
        ref_rule = {"workload": "amr_ldc2d_128_log2", "coarse_steps": n_t, "ms": ms_tot,
                    "value": cells / (ms_tot * 1e-3) / 1e6, "blocks_per_level": c.counts()["n_ids"][:-1],
                    "timed_like": "the reference harness: coarse steps after the spin-up, no refinement turn"}
        c.close()

    # --- end to end through the C ABI with host buffers ----------------------
    e2e = e2e_timed(a.workload, head["tune"]["variant"], a.steps)

    # --- roofline of the fused step kernel on large cases --------------------
    roofline = roofline_of(a.roofline_workload or ROOFLINE_FOR.get(w["storage"], "ldc2d_8192"))
    roofline_fp32 = roofline_of(ROOFLINE_FOR[_lib.STORE_FP32]) if w["storage"] != _lib.STORE_FP32 else None

    # --- precision: FP32 / FP16 against FP64 on the headline case ----------
    errors = error_vs_fp64(a.workload, a.error_steps, local) if (a.error_steps > 0 and w.get("amr")) else None
    channel = config4(torch, local, a.config4_steps) if a.config4_steps > 0 else None

    # --- batched independent cases vs the same cases one at a time -----------
    batched = None
    if a.batched_cases > 0:
        batched = run_batched(torch, a.batched_cases, a.batched_seed, spinup=40, steps=20, device=local,
                              rank=rank, ws=ws, allsum=allsum, allmax=allmax, barrier=barrier)

    # --- CPU baseline (rank 0 only) -------------------------------------------
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = run_cpu_oracle(w, seconds=a.cpu_seconds, threads=threads)

    if ws > 1:
        dist.destroy_process_group()
    if rank == 0:
        extra = {"parallelism": f"replicas x{ws}",
                 "l2": "flushed before every timed step" if head["flush"] else "inputs larger than L2",
                 "autotune": head["tune"], "blocks_per_level": head["counts"]["n_ids"][:-1],
                 "cell_updates_per_step": head["cells_per_step"], "regrids_timed": head["regrids"],
                 "ms_per_coarse_step": head["ms_per_coarse_step"]}
        line = dict(base, value=head["value"], ms_per_step=head["ms_per_step"],
                    config=config_of(a.workload, extra), e2e=e2e, roofline=roofline, cpu_baseline=cpu,
                    clocks=head["clocks"], gpu_launches=head["launches"])
        if roofline_fp32 is not None:
            line["roofline_fp32"] = roofline_fp32
        if plain is not None:
            line["plain_fp32"] = {"workload": a.plain_workload, "value": plain["value"],
                                  "ms_per_step": plain["ms_per_step"], "regrids_timed": plain["regrids"],
                                  "blocks_per_level": plain["counts"]["n_ids"][:-1],
                                  "ratio": head["value"] / plain["value"]}
        if learned is not None:
            line["learned"] = learned
        if ref_rule is not None:
            line["reference_rule_fp32"] = ref_rule
        if errors is not None:
            line["error_vs_fp64"] = errors
        if channel is not None:
            line["channel_d3q27"] = channel
        if batched is not None:
            line["batched"] = batched
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
