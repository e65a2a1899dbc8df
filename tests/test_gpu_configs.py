"""Parity and precision at the benchmark configurations.

* Plain method, 256^2 D2Q9 cavity at Re 100, 10,000 FP32 steps: the
  reference's own CUDA build (oracle/_ref, run here when it was built)
  against this library: integer arrays bit-exact, rho and u within the
  reference's own FP32 floor (its distance from this library's FP64 run),
  centreline profiles u(y) at x = 1/2 and v(x) at y = 1/2 to 5e-6; FP16
  weight-offset storage within 1e-3 (relative L2 of u) of FP64.
* D3Q19 MRT cavity, 128^3 base in 4^3 blocks, 2 levels (boundary-block
  refinement), Re 400, s_nu from Re and the other rates 1.2, 5,000 coarse
  steps: the mesh bit-exact against the CPU oracle (the reference's CUDA
  build faults at this size: an illegal memory access in its near-wall pass
  once its pool has taken 97.5% of free memory), and FP32 / FP16 / BF16 u
  and rho against FP64 on the same mesh.
* The 3-level 128^2 cavity at Re 1000 with the percentile rule: FP32 and
  FP16 against FP64 over 20,000 coarse steps on one mesh (the FP64 run's
  after its 1,280-step spin-up; each storage then continues from that state
  without regrids, so the comparison is of storage, not of refinement
  decisions).
* Drag and lift of a tilted ellipsoid (D3Q19, 64^3, two near-wall levels,
  interpolated bounce-back, second-order momentum exchange, Re 100): FP16
  and FP32 within 1% of FP64.
"""
import json
import tempfile
from pathlib import Path

import numpy as np
import pytest

from helpers import lattice, macros_from_F, rel_l2
from test_oracle import compare_ints, params_for_golden

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def leaf_fields(case, p, Q, dim):
    """rho, u of every active block's cells (sorted block IDs)."""
    nmb, MC = p.n_maxcblocks, 4 ** dim
    cnt = case.counts()
    ids = case.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    blocks = np.sort(np.concatenate([ids[L, :cnt["n_ids"][L]] for L in range(cnt["max_levels"])])).astype(np.int64)
    F = case.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks, :].reshape(Q, -1)
    pb, c, _ = lattice(Q)
    rho, u = macros_from_F(F, dim, Q, pb, c)
    return rho, np.stack(u), blocks


def copy_state(src, dst):
    """Every mesh array, the populations and the counts of src into dst."""
    for arr in (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_F_X, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR,
                _lib.ARR_CBLOCK_ID_NBR_CHILD, _lib.ARR_CBLOCK_ID_ONB, _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL,
                _lib.ARR_ID_SET, _lib.ARR_GAP_SET, _lib.ARR_F):
        dst.load(arr, src.dump(arr))
    cnt = src.counts()
    dst.set_counts(cnt["n_ids"], cnt["id_max"], cnt["n_gaps"])


def test_config1_ldc256_10k_steps_vs_reference_build():
    from oracle.ref_run import REF_BIN, run_ref
    if not (REF_BIN / "ref_d2q9_ldc").exists():
        pytest.skip("the reference's CUDA build (oracle/_ref) was not built")
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_golden import read_dump
    keys = dict(Nx=256, v0=5e-4)
    steps = 10000
    with tempfile.TemporaryDirectory() as td:
        raw = Path(td) / "c1.bin"
        run_ref("ref_d2q9_ldc", keys, steps, 4096, raw)
        g = read_dump(raw)
    g["case_keys"] = json.dumps(keys)
    g["binary"] = "ref_d2q9_ldc"
    p, n = params_for_golden(g)
    assert n == steps
    blocks = g["blocks"].astype(np.int64)
    pb, cv, _ = lattice(9)
    Fr = np.transpose(g["F"][:, :9, :], (1, 0, 2)).reshape(9, -1).astype(np.float64)
    rho_r, u_r = macros_from_F(Fr, 2, 9, pb, cv)
    u_r = np.stack(u_r)
    fields = {}
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
        p.storage = st
        with ag.Case(p) as c:
            c.set_ic(0)
            c.advance_n(steps, use_graph=True)
            c.sync()
            if name == "fp32":
                compare_ints(g, c.dump, c.counts())
            F = c.dump(_lib.ARR_F).reshape(9, p.n_maxcblocks, 16)[:, blocks, :].reshape(9, -1)
            rho, u = macros_from_F(F, 2, 9, pb, cv)
            fields[name] = (rho, np.stack(u))
    rho64, u64 = fields["fp64"]
    rho32, u32 = fields["fp32"]
    floor_u, floor_rho = rel_l2(u_r, u64), rel_l2(rho_r, rho64)
    e_u, e_rho = rel_l2(u32, u_r), rel_l2(rho32, rho_r)
    print(f"\nconfig 1: FP32 vs reference u {e_u:.2e} rho {e_rho:.2e}; reference vs FP64 u {floor_u:.2e}")
    assert e_u < max(1e-5, 2 * floor_u) and e_rho < max(1e-5, 2 * floor_rho)
    assert rel_l2(u32, u64) <= 1.5 * floor_u + 1e-7

    def grid(v):
        a = np.zeros((256, 256))
        bx, by = blocks % 64, blocks // 64
        vv = v.reshape(len(blocks), 16)
        for k in range(16):
            a[by * 4 + k // 4, bx * 4 + k % 4] = vv[:, k]
        return a

    def centrelines(u):
        U, V = grid(u[0]), grid(u[1])
        return 0.5 * (U[:, 127] + U[:, 128]), 0.5 * (V[127, :] + V[128, :])

    pu_r, pv_r = centrelines(u_r)
    pu, pv = centrelines(u32)
    assert np.abs(pu - pu_r).max() < 5e-6 and np.abs(pv - pv_r).max() < 5e-6
    e16 = rel_l2(fields["fp16"][1], u64)
    print(f"config 1: FP16 vs FP64 u {e16:.2e}")
    assert e16 < 1e-3


def test_config3_mrt128_two_levels_mesh_and_precision():
    from oracle.orc import OracleCase
    base = dict(velocity_set=_lib.D3Q19, Nx=128, v0=1.25e-4, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1,
                region_preset=_lib.REGION_BOUNDARY, bc_preset=_lib.BC_LDC3D, collision=_lib.MRT,
                s1=1.2, s2=1.2, s3=1.2, s4=1.2, s5=1.2, s6=1.2, n_maxcblocks=32768 + 46144 + 64)
    p = ag.default_params(**base)
    o = OracleCase(p, p.n_maxcblocks)
    o.set_ic(0)
    o.refine_near_wall()
    fields = {}
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16),
                     ("bf16", _lib.STORE_BF16)):
        p = ag.default_params(storage=st, **base)
        with ag.Case(p) as c:
            c.set_ic(0)
            c.refine_near_wall()
            c.sync()
            if name == "fp64":
                cc, oc = c.counts(), o.counts()
                assert cc["n_ids"] == oc["n_ids"] and cc["id_max"] == oc["id_max"] and cc["n_gaps"] == oc["n_gaps"]
                assert cc["n_ids"][:2] == [32768, 46144]
                for k in (_lib.ARR_CBLOCK_ID_NBR, _lib.ARR_CBLOCK_ID_NBR_CHILD, _lib.ARR_CBLOCK_ID_MASK,
                          _lib.ARR_CBLOCK_ID_ONB, _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL, _lib.ARR_ID_SET,
                          _lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_F_X):
                    assert np.array_equal(c.dump(k), o.dump(k)), k
            c.advance_n(5000, use_graph=True)
            c.sync()
            fields[name] = leaf_fields(c, p, 19, 3)
    o.close()
    r64, u64, b64 = fields["fp64"]
    bars = {"fp32": 1e-3, "fp16": 1e-3, "bf16": 5e-3}
    for name, bar in bars.items():
        r, u, b = fields[name]
        assert np.array_equal(b, b64)
        eu, er = rel_l2(u, u64), rel_l2(r, r64)
        print(f"\nconfig 3: {name} vs FP64 after 5,000 steps: u {eu:.2e} rho {er:.2e}")
        assert eu < bar and er < bar * 1e-1


def test_config2_fp32_fp16_vs_fp64_20k_steps_one_mesh():
    import bench
    w = bench.WORKLOADS["amr_ldc2d_128"]
    p64 = bench.make_params(dict(w, storage=_lib.STORE_FP64), device=0)
    fields = {}
    with ag.Case(p64) as s:
        s.set_ic(0)
        s.refine_near_wall()
        s.advance_n(w["spinup"], use_graph=True)
        s.sync()
        for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
            p = bench.make_params(dict(w, storage=st), device=0, P_REFINE=10 ** 8)
            with ag.Case(p) as c:
                copy_state(s, c)
                c.advance_n(20000 - w["spinup"], use_graph=True)
                c.sync()
                fields[name] = leaf_fields(c, p, 9, 2)
    r64, u64, b64 = fields["fp64"]
    for name, bar in (("fp32", 1e-3), ("fp16", 1e-3)):
        r, u, b = fields[name]
        assert np.array_equal(b, b64)
        eu, er = rel_l2(u, u64), rel_l2(r, r64)
        print(f"\nconfig 2: {name} vs FP64, 20,000 coarse steps: u {eu:.2e} rho {er:.2e}")
        assert eu < bar and er < bar


def test_drag_lift_fp16_within_one_percent():
    from agal_b200.geometry import icosphere
    f = icosphere(3, 1.0, (0, 0, 0), seed=9).astype(np.float64)
    th = 0.35
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    f = ((f * np.array([0.16, 0.07, 0.08])) @ R.T + np.array([0.42, 0.5, 0.5])).astype(np.float32)
    forces = {}
    for name, st in (("fp64", _lib.STORE_FP64), ("fp32", _lib.STORE_FP32), ("fp16", _lib.STORE_FP16)):
        p = ag.default_params(velocity_set=_lib.D3Q19, Nx=64, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1,
                              v0=0.05 * 0.32 / 100, P_REFINE=10 ** 8, G_BIN_DENSITY=8, G_BIN_LEVELS=2, G_BIN_SPEC=2,
                              G_BIN_MAKE_LINKS=1, G_NEAR_WALL_DISTANCE=0.05, S_BC_TYPE=1, S_FORCE_TYPE=0,
                              S_FORCE_ORDER=2, bc_preset=_lib.BC_FPSC3D, ic_preset=_lib.IC_UNIFORM, u_ref=0.05,
                              storage=st, n_maxcblocks=4096 * 4 + 64)
        with ag.Case(p) as c:
            c.set_geometry(f)
            c.set_ic(0)
            c.refine_near_wall()
            c.advance_n(2999, use_graph=True)
            c.forces()   # reset the partials: the next step's sums alone
            c.advance_n(1, use_graph=True)
            fr = c.forces()
            forces[name] = np.array([fr[0] - fr[1], fr[2] - fr[3], fr[4] - fr[5]])
    F64 = forces["fp64"]
    assert abs(F64[1]) > 0.1 * abs(F64[0])   # the tilted body carries lift
    for name in ("fp32", "fp16"):
        d = abs(forces[name][0] - F64[0]) / abs(F64[0])
        lft = abs(forces[name][1] - F64[1]) / abs(F64[1])
        print(f"\ndrag/lift {name} vs FP64: {d:.2e} / {lft:.2e}")
        assert d < 0.01 and lft < 0.01
