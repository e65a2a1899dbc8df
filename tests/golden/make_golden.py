#!/usr/bin/env python
"""Generate the golden fixtures that pin the oracle and the CUDA library to
the reference (KhodrJ/AGAL).

    python tests/golden/make_golden.py tables [--ref DIR]   (default: $AGAL_REFERENCE_DIR)
        Extract the lattice tables (direction vectors, opposites, neighbour
        slot map, weights, block-neighbour directions) from the reference
        sources (inc/util.h:94-101, src/solver_lbm/solver_lbm_init.cu:79-91,
        inc/mesh.h:468-472) into lattice_tables.json.  CPU only; needs the
        reference tree.

    python tests/golden/make_golden.py ref --out DIR
        Run the reference's own CUDA build (oracle/_ref/ref_*, built by
        `make -C oracle ref`) on the cases of CASES and convert each binary
        dump into DIR/<case>.npz.  Needs a GPU; the reference tree is not
        needed at run time.

    python tests/golden/make_golden.py time --out DIR
        Time the reference CUDA build (MLUPS, CUDA events around its
        M_Advance_Step loop) on the benchmark workloads; writes DIR/ref_timing.json.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from oracle.ref_run import BASE_KEYS, REF_BIN, run_ref, write_input  # noqa: E402,F401

# Golden cases: (binary, input.txt keys, steps, keep_mb).  keep_mb is the free
# device memory the reference sizes its block pool from; it must leave room
# for the 2 MB granularity of its ~25 separate allocations.
CASES = {
    "d2q9_ldc64_re100": ("ref_d2q9_ldc", dict(Nx=64, v0=5e-4), 1000, 4096),
    "d2q9_ldc64_px": ("ref_d2q9_ldc", dict(Nx=64, v0=5e-4, PERIODIC_X=1), 300, 4096),
    "d2q9_ldc32x64": ("ref_d2q9_ldc", dict(Nx=32, L_fy=2.0, v0=5e-4), 300, 4096),
    "d3q19_ldc16_re400": ("ref_d3q19_ldc", dict(Nx=16, v0=1.25e-4), 200, 4096),
    "d3q27_ldc16_re200": ("ref_d3q27_ldc", dict(Nx=16, v0=2.5e-4), 200, 4096),
    "d3q19_ldc16_pxy": ("ref_d3q19_ldc", dict(Nx=16, v0=1.25e-4, PERIODIC_X=1, PERIODIC_Y=1), 100, 4096),
    # LES (one level): the field carries the eddy viscosity in row Q + 4.
    "les_d3q19_ldc16_smag": ("ref_d3q19_ldc_smag", dict(Nx=16, v0=1.25e-4), 200, 4096),
    "les_d3q19_ldc16_wale": ("ref_d3q19_ldc_wale", dict(Nx=16, v0=1.25e-4), 200, 4096),
    "les_d3q19_ldc16_vreman": ("ref_d3q19_ldc_vreman", dict(Nx=16, v0=1.25e-4), 200, 4096),
    # 2D models (the N_DIM == 2 branches of solver_lbm_kernels_les.cu:35-213)
    "les_d2q9_ldc64_smag": ("ref_d2q9_ldc_smag", dict(Nx=64, v0=2.5e-5), 400, 4096),
    "les_d2q9_ldc64_wale": ("ref_d2q9_ldc_wale", dict(Nx=64, v0=2.5e-5), 400, 4096),
    "les_d2q9_ldc64_vreman": ("ref_d2q9_ldc_vreman", dict(Nx=64, v0=2.5e-5), 400, 4096),
}

# Multi-level cases: (binary, keys, steps, keep_mb, region preset of the
# Cu_RefineRegion hook (REF_REGION: 0 none, 1 boundary blocks, 2 box)).
# Near-wall/region refinement builds a static hierarchy before the loop;
# MAX_LEVELS_INTERIOR > 1 adds the solution criterion every P_REFINE steps.
AMR = dict(MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, P_REFINE=16, N_REFINE_START=-2.0, N_REFINE_INC=1.0,
           N_REFINE_MAX=1.0, S_CRITERION=0)
AMR_CASES = {
    "amr_d2q9_box3_cubic": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-4, MAX_LEVELS_WALL=3), 200, 4096, 2),
    "amr_d2q9_wall2_linear": ("ref_d2q9_ldc_lin", dict(AMR, Nx=64, v0=5e-4, MAX_LEVELS_WALL=2), 200, 4096, 1),
    # No cubic solution-refinement trajectory: the reference evaluates its cubic
    # interpolant in FP32 from monomial coefficients (util_interp.h), whose
    # rounding (1e-5..1e-4 per interpolation) moves the flow far more than
    # FP32 round-off does, so vorticity near a criterion threshold decides
    # differently from any accurate evaluation within a few regrids.  The
    # regrid pairs below check cubic refinement on identical inputs instead.
    "amr_d2q9_sol3_linear": ("ref_d2q9_ldc_lin", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_INTERIOR=3), 200, 4096, 0),
    "amr_d2q9_wall2_sol3": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=3),
                            200, 4096, 1),
    "amr_d3q19_box2": ("ref_d3q19_ldc", dict(AMR, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=2), 60, 4096, 2),
    "amr_d3q27_sol2": ("ref_d3q27_ldc", dict(AMR, Nx=16, v0=2.5e-5, MAX_LEVELS_INTERIOR=2, P_REFINE=8), 48, 4096, 0),
    # Multi-level LES: the eddy viscosity reads the macro rows as the
    # transfers and collides leave them; the field's rows Q..Q+dim hold the
    # last macros, row Q+4 the last eddy viscosity.
    "les_d2q9_wall2_smag_lin": ("ref_d2q9_ldc_smag_lin", dict(AMR, Nx=64, v0=2.5e-5, MAX_LEVELS_WALL=2), 400, 4096,
                                1),
    "les_d3q19_box2_wale": ("ref_d3q19_ldc_wale", dict(AMR, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=2), 100, 4096, 2),
    "les_d2q9_sol2_vreman_lin": ("ref_d2q9_ldc_vreman_lin", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_INTERIOR=2),
                                 160, 4096, 0),
}

# Regrid pairs: the reference state just before the refinement of the last
# step (<name>_pre) and right after it (<name>_post).  Loading the first and
# refining must give the second bit for bit: the criterion, marks and the
# refine/coarsen pass judged on identical inputs, whatever FP32 rounding did to
# the trajectory before.  (binary, keys, steps, keep_mb, region)
REGRID_PAIRS = {
    "regrid_d2q9_cubic_s128": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_INTERIOR=3), 128, 4096, 0),
    "regrid_d2q9_cubic_s48": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_INTERIOR=3), 48, 4096, 0),
    "regrid_d2q9_linear_s64": ("ref_d2q9_ldc_lin", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_INTERIOR=3), 64, 4096, 0),
    "regrid_d2q9_wall_s96": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=3),
                             96, 4096, 1),
    "regrid_d3q19_s24": ("ref_d3q19_ldc", dict(AMR, Nx=16, v0=2.5e-5, MAX_LEVELS_INTERIOR=2, P_REFINE=8), 24, 4096, 0),
    "regrid_d3q27_s40": ("ref_d3q27_ldc", dict(AMR, Nx=16, v0=2.5e-5, MAX_LEVELS_INTERIOR=2, P_REFINE=8), 40, 4096, 0),
}

# Geometry cases: a seeded icosphere (agal_b200.geometry.icosphere) written as
# ASCII STL into the case's geometry/ folder, imported, binned and voxelized by
# the reference (REF_GEOM=1), then flow past it with the custom.h FPSC-3D
# preset.  The dump adds the faces, bins, link lengths and MEA partials.
# (binary, keys, steps, keep_mb, sphere: subdivisions, radius, centre, seed)
# The domain is the unit cube: the reference's ray filter and bin lookups
# index cells as coordinate x N (geometry_bins_gpu.cu:203-206,
# mesh_voxelizer_voxelize.cu:253-258), which is only right when every side
# has length 1.
GEO = dict(AMR, L_fy=1.0, L_fz=1.0, G_LOADTYPE=0, G_FILENAME="sphere.stl", G_BIN_DENSITY=8, G_BIN_LEVELS=3,
           G_BIN_SPEC=2, G_BIN_APPROACH=1, G_BIN_MAKE_LINKS=1, G_NEAR_WALL_DISTANCE=0.05, G_VIS_TREE=0, G_PRINT=0,
           P_REFINE=100000, S_FORCE_TYPE=0)
GEOM_CASES = {
    "geom_d3q19_wall3_bouzidi": ("ref_d3q19_fps", dict(GEO, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=3, MAX_LEVELS_INTERIOR=3,
                                                       S_BC_TYPE=1, S_FORCE_ORDER=2), 24, 4096,
                                 (3, 0.07, (0.45, 0.5, 0.5), 7)),
    "geom_d3q27_wall2_bb": ("ref_d3q27_fps", dict(GEO, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=2,
                                                  G_BIN_LEVELS=2, S_BC_TYPE=0, S_FORCE_ORDER=1), 16, 4096,
                            (3, 0.1, (0.46, 0.49, 0.51), 11)),
    "geom_d3q19_cv": ("ref_d3q19_fps", dict(GEO, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=3, MAX_LEVELS_INTERIOR=3,
                                            S_BC_TYPE=1, S_FORCE_TYPE=1, S_FORCEVOLUME_Xm=0.28,
                                            S_FORCEVOLUME_XM=0.66, S_FORCEVOLUME_Ym=0.31, S_FORCEVOLUME_YM=0.69,
                                            S_FORCEVOLUME_Zm=0.3, S_FORCEVOLUME_ZM=0.7), 16, 4096,
                      (3, 0.07, (0.45, 0.5, 0.5), 7)),
    # LES (Smagorinsky) with the interpolated bounce-back on a two-level mesh:
    # the field carries the macro rows and the eddy viscosity row.
    "geom_les_d3q19_wall2_smag": ("ref_d3q19_fps_smag", dict(GEO, Nx=16, v0=1.25e-4, MAX_LEVELS_WALL=2,
                                                             MAX_LEVELS_INTERIOR=2, G_BIN_LEVELS=2, S_BC_TYPE=1,
                                                             S_FORCE_ORDER=2), 40, 4096,
                                  (3, 0.1, (0.46, 0.49, 0.51), 11)),
    "geom_d3q19_uniform": ("ref_d3q19_fps", dict(GEO, Nx=32, v0=1.25e-4, G_BIN_DENSITY=16, G_BIN_LEVELS=1,
                                                 MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, S_BC_TYPE=1,
                                                 S_FORCE_ORDER=2), 20, 4096, (3, 0.15, (0.47, 0.52, 0.49), 3)),
}

# Timing workloads of the reference build: (binary, keys, timed steps, keep_mb)
TIMING = {
    "ldc2d_256": ("ref_d2q9_ldc", dict(Nx=256, v0=5e-4), 2000, 4096),
    "ldc2d_8192": ("ref_d2q9_ldc", dict(Nx=8192, v0=5e-4), 20, 16384),
    "ldc3d19_384": ("ref_d3q19_ldc", dict(Nx=384, v0=1.25e-4), 10, 24576),
}



# ---------------------------------------------------------------------------
def _c_array(text: str, name: str) -> list[float]:
    m = re.search(name + r"\s*\[[^\]]*\]\s*=\s*\{([^}]*)\}", text)
    if not m:
        raise ValueError(f"array {name} not found")
    out = []
    for tok in m.group(1).split(","):
        tok = tok.strip()
        if not tok:
            continue
        if "/" in tok:
            a, b = tok.split("/")
            out.append(float(a) / float(b))
        else:
            out.append(float(tok))
    return out


def cmd_tables(ref: Path) -> None:
    util = (ref / "inc" / "util.h").read_text()
    init = (ref / "src" / "solver_lbm" / "solver_lbm_init.cu").read_text()
    mesh = (ref / "inc" / "mesh.h").read_text()
    t = {}
    for nm in ["V_CONN_ID_2D", "V_CONN_ID_3D", "V_CONN_ID_PB_2D", "V_CONN_ID_PB_3D", "V_CONN_MAP_2D", "V_CONN_MAP_3D"]:
        t[nm] = [int(v) for v in _c_array(util, nm)]
    for nm in ["LBMw_D2Q9", "LBMw_D3Q19", "LBMw_D3Q27"]:
        t[nm] = _c_array(init, nm)
    for nm in ["LBMpb_D2Q9", "LBMpb_D3Q19", "LBMpb_D3Q27"]:
        t[nm] = [int(v) for v in _c_array(init, nm)]
    m = re.search(r"c\[2\]\[27\*3\]\s*=\s*\{(.*?)\};", mesh, re.S)
    rows = re.findall(r"\{([^{}]*)\}", m.group(1))
    t["MESH_C_2D"] = [int(float(v)) for v in rows[0].split(",") if v.strip()]
    t["MESH_C_3D"] = [int(float(v)) for v in rows[1].split(",") if v.strip()]
    (HERE / "lattice_tables.json").write_text(json.dumps(t, indent=1))
    print("wrote", HERE / "lattice_tables.json")


# ---------------------------------------------------------------------------
LES_BINARIES = ("ref_d3q19_ldc_smag", "ref_d3q19_ldc_wale", "ref_d3q19_ldc_vreman",
                "ref_d2q9_ldc_smag", "ref_d2q9_ldc_wale", "ref_d2q9_ldc_vreman", "ref_d2q9_ldc_smag_lin",
                "ref_d2q9_ldc_vreman_lin", "ref_d3q19_fps_smag")


def read_dump(path: Path, les: bool = False) -> dict:
    """Parse an AGALREF1 dump written by oracle/ref_harness/ref_main.cu (an LES
    build's field has one more row, the eddy viscosity)."""
    b = path.read_bytes()
    if b[:8] != b"AGALREF1":
        raise ValueError("bad magic")
    o = 8

    def take(dt, n):
        nonlocal o
        a = np.frombuffer(b, dtype=dt, count=n, offset=o).copy()
        o += a.nbytes
        return a

    dim, Q, Qmax, MC, ML, steps = take(np.int32, 6)
    nmb, nmc = take(np.int64, 2)
    n_ids = take(np.int32, ML + 1)
    id_max = take(np.int32, ML + 1)
    n_gaps = take(np.int32, 1)[0]
    id_sets = [take(np.int32, int(n_ids[L])) for L in range(ML)]
    n_gap_keep = take(np.int32, 1)[0]
    gaps_tail = take(np.int32, int(n_gap_keep))
    n_act = take(np.int32, 1)[0]
    blocks = take(np.int32, int(n_act))
    NU = Q + 5 if les else Q + dim + 1   # the harness sizes LES fields N_Q + 5 (eddy viscosity in row N_Q + 4)
    rec = [("fX", np.float32, dim), ("bmask", np.int32, 1), ("nbr", np.int32, Qmax), ("nbr_child", np.int32, Qmax),
           ("onb", np.int32, 1), ("ref", np.int32, 1), ("level", np.int32, 1), ("cmask", np.int32, MC),
           ("F", np.float32, NU * MC)]
    out = {k: [] for k, _, _ in rec}
    for _ in range(int(n_act)):
        for k, dt, n in rec:
            out[k].append(take(dt, n))
    res = dict(dim=int(dim), Q=int(Q), Qmax=int(Qmax), MC=int(MC), max_levels=int(ML), steps=int(steps),
               n_maxcblocks=int(nmb), n_maxcells=int(nmc), n_ids=n_ids, id_max=id_max, n_gaps=int(n_gaps),
               gaps_tail=gaps_tail, blocks=blocks)
    for L in range(ML):
        res[f"id_set_{L}"] = id_sets[L]
    for k, _, _ in rec:
        res[k] = np.stack(out[k]) if out[k] else np.zeros((0,))
    res["F"] = res["F"].reshape(int(n_act), NU, int(MC))
    if o < len(b) and b[o:o + 4] == b"GEOM":
        o += 4
        nf = int(take(np.int64, 1)[0])
        res["faces_soa"] = take(np.float32, 9 * nf).reshape(9, nf)
        nbl = int(take(np.int32, 1)[0])
        res["n_bin_levels"] = nbl
        for L in range(nbl):
            dens, nb = (int(v) for v in take(np.int32, 2))
            ne = int(take(np.int64, 1)[0])
            res[f"bins_density_{L}"] = dens
            res[f"bins_n_{L}"] = take(np.int32, nb)
            res[f"bins_N_{L}"] = take(np.int32, nb)
            res[f"bins_ids_{L}"] = take(np.int32, ne)
        mk = int(take(np.int32, 1)[0])
        res["make_links"] = mk
        if mk:
            lmd, dens, nb = (int(v) for v in take(np.int32, 3))
            ne = int(take(np.int64, 1)[0])
            res["bins_md_level"] = lmd
            res["bins_md_density"] = dens
            res["bins_md_n"] = take(np.int32, nb)
            res["bins_md_N"] = take(np.int32, nb)
            res["bins_md_ids"] = take(np.int32, ne)
        sa, sb, mcb = (int(v) for v in take(np.int64, 3))
        res["n_solida"], res["n_solidb"], res["n_maxcells_b"] = sa, sb, mcb
        if sb > 0:
            res["onb_solid"] = take(np.int32, int(n_act))
        nxb = int(take(np.int64, 1)[0])
        if nxb:
            res["cells_f_X_b"] = take(np.float32, nxb).reshape(int(Qmax), mcb)
        res["Ff"] = take(np.float32, 6 * int(n_act)).reshape(int(n_act), 6)
    return res


def cmd_ref(out: Path, only: list[str] | None) -> None:
    out.mkdir(parents=True, exist_ok=True)
    cases = {k: v + (0, False, None) for k, v in CASES.items()}
    cases.update({k: v + (False, None) for k, v in AMR_CASES.items()})
    for k, v in REGRID_PAIRS.items():
        cases[k + "_pre"] = v + (True, None)
        cases[k + "_post"] = v + (False, None)
    for k, (binary, keys, steps, keep, sphere) in GEOM_CASES.items():
        cases[k] = (binary, keys, steps, keep, 0, False, sphere)
    # Multi-level geometry fixtures keep the populations of the wall blocks
    # only (blocks with a solid-boundary slot); the uniform one keeps all.
    wall_only_F = {"geom_d3q19_wall3_bouzidi", "geom_d3q27_wall2_bb", "geom_d3q19_cv"}
    for name, (binary, keys, steps, keep, region, skip, sphere) in cases.items():
        if only and not any(name == o or name.startswith(o + "_") for o in only):
            continue
        raw = out / f"{name}.bin"
        run_ref(binary, keys, steps, keep, raw, region=region, skip_last_regrid=skip, sphere=sphere)
        d = read_dump(raw, les=binary in LES_BINARIES)
        d["case_keys"] = json.dumps(keys)
        d["binary"] = binary
        d["region"] = region
        if sphere is not None:
            d["sphere"] = json.dumps(sphere)
            if name in wall_only_F:
                keep_blk = d["onb_solid"] >= 0
                d["F_blocks"] = np.nonzero(keep_blk)[0].astype(np.int32)
                d["F"] = d["F"][keep_blk]
        np.savez_compressed(out / f"{name}.npz", **d)
        raw.unlink()
        print(name, "n_maxcblocks", d["n_maxcblocks"], "active", len(d["blocks"]), flush=True)


# Restart fixture: the reference's own restart.bin of an AMR run (near-wall
# and solution refinement), with a small memory allowance so that the block
# pool, and with it the gap stack in the file, stays small; the harness dump
# of the same state goes beside it.
RESTART_CASES = {
    "restart_d2q9_wall2_sol3": ("ref_d2q9_ldc", dict(AMR, Nx=64, v0=5e-5, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=3,
                                                      N_PRINT_LEVELS=2, VOL_I_MIN=0, VOL_I_MAX=64, VOL_J_MIN=0,
                                                      VOL_J_MAX=64, N_ITER_TOTAL=200, P_OUTPUT=100,
                                                      N_OUTPUT_START=0), 200, 4096),
}


def cmd_restart(out: Path) -> None:
    out.mkdir(parents=True, exist_ok=True)
    for name, (binary, keys, steps, keep) in RESTART_CASES.items():
        raw, rbin, ubin = out / f"{name}.bin", out / f"{name}.restart", out / f"{name}.uniform"
        run_ref(binary, keys, steps, keep, raw, restart=rbin, uniform=ubin)
        d = read_dump(raw)
        d["case_keys"] = json.dumps(keys)
        d["binary"] = binary
        b = rbin.read_bytes()
        # The gap stack (most of the file: the untouched part of the pool's
        # descending ID list) is kept as first value + differences; the bytes
        # before and after it verbatim; the file's SHA-256 checks the rebuild.
        ml = int(d["max_levels"])
        head = np.frombuffer(b, dtype=np.int32, count=2 * (ml + 1) + 5 + 2)
        n_ids, n_gaps = head[1:ml + 2], int(head[ml + 2])
        g0 = 4 * (2 * (ml + 1) + 5) + 8 + 4 * int(n_ids[:ml].sum())
        gaps = np.frombuffer(b, dtype=np.int32, count=n_gaps, offset=g0)
        d["restart_head"] = np.frombuffer(b[:g0], dtype=np.uint8)
        d["restart_gap_first"] = np.int32(gaps[0] if n_gaps else 0)
        d["restart_gap_diff"] = np.diff(gaps).astype(np.int32)
        d["restart_n_gaps"] = n_gaps
        d["restart_tail"] = np.frombuffer(b[g0 + 4 * n_gaps:], dtype=np.uint8)
        d["restart_sha256"] = hashlib.sha256(b).hexdigest()
        d["out_direct"] = np.frombuffer(ubin.read_bytes(), dtype=np.uint8)
        np.savez_compressed(out / f"{name}.npz", **d)
        raw.unlink()
        rbin.unlink()
        ubin.unlink()
        print(name, "n_maxcblocks", d["n_maxcblocks"], "restart bytes", len(b), flush=True)


# Face import fixtures: the reference's face list after its import and the
# splitting of long faces (G_Init_Arrays_CoordsList_CPU) for a coarse STL
# icosphere whose faces get split, and for the primitives of a geometry.txt.
FACE_CASES = {
    "faces_stl_split": (dict(GEO, Nx=16, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, G_BIN_LEVELS=1, G_BIN_DENSITY=16),
                        (1, 0.3, (0.5, 0.5, 0.5), 5), None),
    "faces_text_primitives": (dict(GEO, Nx=16, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, G_BIN_LEVELS=1,
                                   G_BIN_DENSITY=8, G_LOADTYPE=1),
                              None, "PRISM CORNER 0.2 0.35 0.3 0.45 0.25 0.4\n"
                                    "PRISM CENTER 0.7 0.6 0.5 0.1 0.15 0.2\n"
                                    "SPHERE 9 13 0.5 0.3 0.6 0.12\nEND\n"),
}


def cmd_faces(out: Path) -> None:
    out.mkdir(parents=True, exist_ok=True)
    for name, (keys, sphere, txt) in FACE_CASES.items():
        raw = out / f"{name}.bin"
        run_ref("ref_d3q19_fps", keys, 1, 4096, raw, sphere=sphere, geometry_txt=txt)
        d = read_dump(raw)
        keep = {k: d[k] for k in ("faces_soa",) if k in d}
        keep["case_keys"] = json.dumps(keys)
        if sphere is not None:
            keep["sphere"] = json.dumps(sphere)
        if txt is not None:
            keep["geometry_txt"] = txt
        np.savez_compressed(out / f"{name}.npz", **keep)
        raw.unlink()
        print(name, "faces", keep["faces_soa"].shape, flush=True)


def cmd_time(out: Path) -> None:
    out.mkdir(parents=True, exist_ok=True)
    res = {}
    for name, (binary, keys, n_timed, keep) in TIMING.items():
        txt = run_ref(binary, keys, 3, keep, None, n_timed=n_timed)
        line = [ln for ln in txt.splitlines() if ln.startswith("{\"ref_timing\"")]
        res[name] = json.loads(line[-1]) if line else {"error": txt[-500:]}
        print(name, res[name], flush=True)
    (out / "ref_timing.json").write_text(json.dumps(res, indent=1))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("tables")
    t.add_argument("--ref", default=os.environ.get("AGAL_REFERENCE_DIR", "/root/reference"))
    r = sub.add_parser("ref")
    r.add_argument("--out", default=str(HERE))
    r.add_argument("--only", nargs="*")
    tm = sub.add_parser("time")
    tm.add_argument("--out", required=True)
    rs = sub.add_parser("restart")
    rs.add_argument("--out", default=str(HERE))
    fc = sub.add_parser("faces")
    fc.add_argument("--out", default=str(HERE))
    a = ap.parse_args(argv)
    if a.cmd == "tables":
        cmd_tables(Path(a.ref))
    elif a.cmd == "ref":
        cmd_ref(Path(a.out).resolve(), a.only)
    elif a.cmd == "restart":
        cmd_restart(Path(a.out).resolve())
    elif a.cmd == "faces":
        cmd_faces(Path(a.out).resolve())
    else:
        cmd_time(Path(a.out).resolve())
    return 0


if __name__ == "__main__":
    sys.exit(main())
