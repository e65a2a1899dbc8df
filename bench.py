#!/usr/bin/env python
"""Benchmark of the B200 octree-AMR lattice Boltzmann time step.

One "step" is one coarse time step of the solver (Solver::S_Advance from
N_LEVEL_START) on the workload named in the JSON line.  Metric: MLUPS
(million lattice-cell updates per second, level-L leaf cells counted 2^(L-L0)
times per coarse step as solver_lbm_advance.cu:74-89 counts them).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl b200 (default): the CUDA library.  Rank 0 prints one JSON line with
  value        device-timed MLUPS (CUDA events on the library's stream, L2
               flushed between steps when the workload fits in L2)
  e2e          MLUPS through the public C ABI with host buffers: load the
               initial populations from pinned host memory, K x (advance +
               read back the FP64 mass/momentum), dump the final populations
  roofline     the fused step kernel on a large case of the same physics
               (inputs far larger than L2), algorithmic bytes 2*Q*s per cell
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

# Workloads (synthetic: initialised at rest, nothing read from disk).
WORKLOADS = {
    "ldc2d_256": dict(
        desc="D2Q9 BGK lid-driven cavity 256x256, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=256, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_256_fp16": dict(
        desc="D2Q9 BGK lid-driven cavity 256x256, one level, Re=100, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D2Q9, Nx=256, Re=100.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC2D),
    "ldc2d_4096": dict(
        desc="D2Q9 BGK lid-driven cavity 4096x4096, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=4096, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_8192": dict(
        desc="D2Q9 BGK lid-driven cavity 8192x8192, one level, Re=100, lid 0.05, FP32 populations",
        velocity_set=_lib.D2Q9, Nx=8192, Re=100.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC2D),
    "ldc2d_8192_fp16": dict(
        desc="D2Q9 BGK lid-driven cavity 8192x8192, one level, Re=100, lid 0.05, FP16 weight-offset populations",
        velocity_set=_lib.D2Q9, Nx=8192, Re=100.0, storage=_lib.STORE_FP16, bc=_lib.BC_LDC2D),
    "ldc3d19_384": dict(
        desc="D3Q19 BGK lid-driven cavity 384^3, one level, Re=400, lid 0.05, FP32 populations",
        velocity_set=_lib.D3Q19, Nx=384, Re=400.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC3D),
    "ldc3d27_256": dict(
        desc="D3Q27 BGK lid-driven cavity 256^3, one level, Re=200, lid 0.05, FP32 populations",
        velocity_set=_lib.D3Q27, Nx=256, Re=200.0, storage=_lib.STORE_FP32, bc=_lib.BC_LDC3D),
}
Q_OF = {_lib.D2Q9: 9, _lib.D3Q19: 19, _lib.D3Q27: 27}
DIM_OF = {_lib.D2Q9: 2, _lib.D3Q19: 3, _lib.D3Q27: 3}
ESIZE = {_lib.STORE_FP32: 4, _lib.STORE_FP64: 8, _lib.STORE_FP16: 2, _lib.STORE_BF16: 2}
DTYPE_NAME = {_lib.STORE_FP32: "f32", _lib.STORE_FP64: "f64", _lib.STORE_FP16: "f16-offset(f32 math)",
              _lib.STORE_BF16: "bf16-offset(f32 math)"}


def make_params(w: dict, device: int = -1):
    dim = DIM_OF[w["velocity_set"]]
    nb = (w["Nx"] // 4) ** dim
    return ag.default_params(
        velocity_set=w["velocity_set"], Nx=w["Nx"], MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1,
        N_LEVEL_START=0, v0=0.05 / w["Re"], bc_preset=w["bc"], ic_preset=_lib.IC_REST,
        storage=w["storage"], n_maxcblocks=nb, device=device)


def cells_per_step(w: dict) -> int:
    return w["Nx"] ** DIM_OF[w["velocity_set"]]


def state_bytes(w: dict) -> int:
    return cells_per_step(w) * Q_OF[w["velocity_set"]] * ESIZE[w["storage"]]


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
def time_steps(case, torch, n_steps: int, flush: bool) -> list[float]:
    """Per-step device time (ms) with CUDA events on the library's stream."""
    stream = torch.cuda.ExternalStream(case.stream_ptr())
    scratch = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda") if flush else None
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
    for i in range(n_steps):
        if flush:
            with torch.cuda.stream(stream):
                scratch.add_(1.0)   # writes 252 MB > L2 between timed steps
        evs[i][0].record(stream)
        case.advance()
        evs[i][1].record(stream)
    case.sync()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in evs]


def run_cpu_oracle(w: dict, seconds: float, threads: int, max_steps: int | None = None) -> dict:
    """Oracle (CPU restatement, OpenMP) MLUPS on a bounded sample of the workload."""
    from oracle.orc import OracleCase, build  # CPU baseline leg only
    build()
    p = make_params(w)
    o = OracleCase(p, p.n_maxcblocks, fp64=(w["storage"] == _lib.STORE_FP64), threads=threads)
    o.set_ic(0)
    t0 = time.perf_counter()
    o.advance_n(2)
    per = (time.perf_counter() - t0) / 2
    n = max(1, int(seconds / max(per, 1e-9)))
    if max_steps:
        n = min(n, max_steps)
    t0 = time.perf_counter()
    o.advance_n(n)
    dt = time.perf_counter() - t0
    o.close()
    mlups = cells_per_step(w) * n / dt / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{n} steps of {w['desc']} on {threads} host threads ({dt:.1f} s)"}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="ldc2d_256", choices=sorted(WORKLOADS))
    ap.add_argument("--roofline-workload", default="ldc2d_8192", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--profile", choices=sorted(WORKLOADS), default=None,
                    help="only run W+K steps of this workload (for ncu captures); prints no JSON line")
    ap.add_argument("--cpt", type=int, default=1, choices=[1, 2, 3],
                    help="with --profile: step kernel variant (1, 2 cells per thread; 3 TMA pipeline)")
    a = ap.parse_args(argv)
    a.warmup = max(a.warmup, 3)
    w = WORKLOADS[a.workload]
    if a.profile:
        pw = WORKLOADS[a.profile]
        with ag.Case(make_params(pw, device=0)) as pc:
            pc.set_ic(0)
            pc.set_tuning(a.cpt)
            for _ in range(a.warmup + a.steps):
                pc.advance()
            pc.sync()
        print(f"profile run done: {a.profile}, {a.warmup}+{a.steps} steps")
        return 0
    ws, rank, local = dist_setup()
    threads = os.cpu_count() or 1
    base = {"metric": "MLUPS (lattice cell updates per second / 1e6), one coarse time step per step",
            "unit": "MLUPS", "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE_NAME[w["storage"]], "data": "synthetic (fluid at rest, lid-driven)"}

    if a.impl == "reference":
        # The reference algorithm on the host cores; other ranks idle.
        if rank != 0:
            return 0
        cb = run_cpu_oracle(w, seconds=1e9, threads=threads, max_steps=a.steps)
        line = dict(base, impl="reference", value=cb["value"], ms_per_step=None,
                    config={"workload": a.workload, "desc": w["desc"], "cells": cells_per_step(w),
                            "parallelism": "host OpenMP", "l2": "n/a (CPU)"},
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

    # --- device-timed steps -------------------------------------------------
    p = make_params(w, device=local)
    case = ag.Case(p)
    case.set_ic(0)
    tune = case.autotune(0, reps=10)
    for _ in range(a.warmup):
        case.advance()
    case.sync()
    flush = state_bytes(w) * 2 < L2_BYTES
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        per_step = time_steps(case, torch, a.steps, flush)
    barrier()
    t_ms = allmax(sum(per_step))
    value = ws * cells_per_step(w) * a.steps / (t_ms * 1e-3) / 1e6
    case.close()

    # --- end to end through the C ABI with host buffers ----------------------
    p = make_params(w, device=local)
    case = ag.Case(p)
    case.set_ic(0)
    case.set_tuning(tune["variant"])
    f0 = case.dump(_lib.ARR_F)
    pinned = torch.from_numpy(f0).pin_memory()
    host_in = pinned.numpy()
    host_out = torch.empty_like(pinned).pin_memory().numpy()
    mm = (C.c_double * 4)()
    lib = _lib.lib()
    barrier()
    t0 = time.perf_counter()
    rc = lib.agal_load(case._h, _lib.ARR_F, host_in.ctypes.data_as(C.c_void_p), host_in.nbytes)
    for _ in range(a.steps):
        rc |= lib.agal_advance(case._h, 0)
        rc |= lib.agal_mass_momentum(case._h, mm)   # D2H of the step's FP64 mass/momentum
    rc |= lib.agal_dump(case._h, _lib.ARR_F, host_out.ctypes.data_as(C.c_void_p), host_out.nbytes)
    e2e_s = time.perf_counter() - t0
    if rc:
        raise RuntimeError("e2e run failed")
    e2e_s = allmax(e2e_s)
    case.close()
    e2e = {"value": ws * cells_per_step(w) * a.steps / e2e_s / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": int(host_in.nbytes / a.steps),
           "d2h_bytes_per_step": int(host_out.nbytes / a.steps) + 8 * (DIM_OF[w["velocity_set"]] + 1)}

    # --- roofline of the fused step kernel on a large case -------------------
    rw = WORKLOADS[a.roofline_workload]
    rp = make_params(rw, device=local)
    rcase = ag.Case(rp)
    rcase.set_ic(0)
    rtune = rcase.autotune(0, reps=5)
    for _ in range(3):
        rcase.advance()
    rcase.sync()
    rsteps = 20
    rt = time_steps(rcase, torch, rsteps, flush=False)
    rcase.close()
    avg_ms = sum(rt) / len(rt)
    alg_bytes = 2 * Q_OF[rw["velocity_set"]] * ESIZE[rw["storage"]] * cells_per_step(rw)
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = dram_traffic_per_launch(a.roofline_workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "kernel": "k_step (fused collide+BC+stream)",
                "workload": a.roofline_workload, "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": avg_ms, "autotune": rtune}

    # --- CPU baseline (rank 0 only) -------------------------------------------
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = run_cpu_oracle(w, seconds=a.cpu_seconds, threads=threads)

    if ws > 1:
        dist.destroy_process_group()
    if rank == 0:
        line = dict(base, value=value, ms_per_step=t_ms / a.steps,
                    config={"workload": a.workload, "desc": w["desc"], "cells": cells_per_step(w),
                            "parallelism": f"replicas x{ws}",
                            "l2": "flushed between timed steps" if flush else "inputs larger than L2",
                            "autotune": tune},
                    e2e=e2e, roofline=roofline, cpu_baseline=cpu, clocks=clk.summary(),
                    gpu_launches=a.steps)
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
