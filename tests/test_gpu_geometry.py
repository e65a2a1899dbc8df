"""The CUDA geometry chain against the reference build's dumps and the oracle.

Per fixture (tests/golden/geom_*.npz, written by the reference's own build):
face bins, voxelized cell and block states, near-wall refinement, wall slots
and FP32 link lengths bit for bit; the flow with the interpolated bounce-back
and the MEA force partials at the FP32 round-off floor of the reference.
FP64 storage against the FP64 oracle within 1e-11 (the same formulas, other
evaluation order).  Step variants and graph replay bit-identical; FP16
storage close to FP64.
"""
import numpy as np
import pytest

from test_oracle import GOLDEN
from test_oracle_geometry import GEOM_CASES, faces_of, geom_params

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu

INT_ARRAYS = (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR, _lib.ARR_CBLOCK_ID_NBR_CHILD,
              _lib.ARR_CBLOCK_ID_ONB, _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL, _lib.ARR_CBLOCK_ID_ONB_SOLID)


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def run_case(g, storage=_lib.STORE_FP32, steps=None, variant=None, use_graph=True):
    p, n = geom_params(g)
    p.storage = storage
    c = ag.Case(p)
    if variant:
        c.set_tuning(variant)
    c.set_geometry(faces_of(g))
    c.set_ic(0)
    c.refine_near_wall()
    c.advance_n(n if steps is None else steps, use_graph=use_graph)
    c.sync()
    return c, p


@pytest.mark.parametrize("name", GEOM_CASES)
def test_cuda_geometry_vs_reference_build(name):
    g = load(name)
    p, steps = geom_params(g)
    c = ag.Case(p)
    c.set_geometry(faces_of(g))
    for L in range(int(g["n_bin_levels"])):
        dens, n, N, ids = c.bins(L)
        assert dens == int(g[f"bins_density_{L}"])
        assert np.array_equal(n, g[f"bins_n_{L}"]) and np.array_equal(N, g[f"bins_N_{L}"]), L
        assert np.array_equal(ids, g[f"bins_ids_{L}"]), L
    dens, n, N, ids = c.bins(-1)
    assert np.array_equal(n, g["bins_md_n"]) and np.array_equal(N, g["bins_md_N"])
    assert np.array_equal(ids, g["bins_md_ids"])
    c.set_ic(0)
    c.refine_near_wall()
    nmb, MC, Qmax, Q = p.n_maxcblocks, int(g["MC"]), int(g["Qmax"]), int(g["Q"])
    blocks = g["blocks"].astype(np.int64)
    ml = int(g["max_levels"])
    assert c.counts()["n_ids"][:ml] == [int(v) for v in g["n_ids"][:ml]]
    assert np.array_equal(c.dump(_lib.ARR_CELLS_ID_MASK).reshape(nmb, MC)[blocks], g["cmask"])
    for arr, key in [(_lib.ARR_CBLOCK_ID_MASK, "bmask"), (_lib.ARR_CBLOCK_ID_REF, "ref"),
                     (_lib.ARR_CBLOCK_ID_ONB, "onb"), (_lib.ARR_CBLOCK_LEVEL, "level")]:
        assert np.array_equal(c.dump(arr)[blocks], g[key][:, 0]), key
    assert np.array_equal(c.dump(_lib.ARR_CBLOCK_ID_NBR).reshape(Qmax, nmb)[:, blocks].T, g["nbr"])
    assert np.array_equal(c.dump(_lib.ARR_CBLOCK_ID_ONB_SOLID)[blocks], g["onb_solid"])
    gc = c.geometry_counts()
    assert (gc["n_solida"], gc["n_solidb"], gc["n_maxcells_b"]) == (int(g["n_solida"]), int(g["n_solidb"]),
                                                                     int(g["n_maxcells_b"]))
    xb = c.dump(_lib.ARR_CELLS_F_X_B).reshape(27, -1)
    assert np.array_equal(xb, g["cells_f_X_b"])
    c.advance_n(steps)
    c.sync()
    fb = blocks[g["F_blocks"]] if "F_blocks" in g else blocks
    F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, fb, :].transpose(1, 0, 2)
    assert np.abs(F - g["F"][:, :Q, :].astype(np.float64)).max() < 2e-6
    Ff = c.dump(_lib.ARR_CBLOCK_F_FF).reshape(6, nmb)[:, blocks].T
    ref = g["Ff"].astype(np.float64)
    assert np.abs(Ff - ref).max() < 5e-6 * np.abs(ref).max()
    sums = c.forces()
    for d in range(3):
        assert abs(sums[2 * d] - ref[:, 2 * d].sum()) < 1e-5 * np.abs(ref[:, 2 * d]).sum() + 1e-12
    assert np.all(c.dump(_lib.ARR_CBLOCK_F_FF) == 0.0)   # reported and reset
    c.close()


@pytest.mark.parametrize("name", GEOM_CASES)
def test_cuda_geometry_fp64_matches_oracle(name):
    from oracle.orc import OracleCase
    g = load(name)
    c, p = run_case(g, storage=_lib.STORE_FP64)
    p2, steps = geom_params(g)
    o = OracleCase(p2, p2.n_maxcblocks, fp64=True)
    o.set_geometry(faces_of(g))
    o.set_ic(0)
    o.refine_near_wall()
    o.advance_n(steps)
    for k in INT_ARRAYS:
        assert np.array_equal(c.dump(k), o.dump(k)), k
    assert np.array_equal(c.dump(_lib.ARR_CELLS_F_X_B), o.dump(_lib.ARR_CELLS_F_X_B))
    nmb, Q, MC = p.n_maxcblocks, int(g["Q"]), int(g["MC"])
    ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    cnt = c.counts()
    blocks = np.sort(np.concatenate([ids[L, : cnt["n_ids"][L]] for L in range(cnt["max_levels"])])).astype(np.int64)
    Fc = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    Fo = o.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    assert np.abs(Fc - Fo).max() < 1e-11
    Ffc, Ffo = c.dump(_lib.ARR_CBLOCK_F_FF), o.dump(_lib.ARR_CBLOCK_F_FF)
    scale = np.abs(Ffo).max()
    assert scale > 0
    assert np.abs(Ffc - Ffo).max() < 1e-11 * scale
    assert np.allclose(c.forces(), o.forces(), rtol=1e-11, atol=1e-11 * scale)
    c.close()


def test_control_volume_forces_vs_reference_build():
    """S_FORCE_TYPE 1 (Cu_ComputeForcesCV) on the 3-level sphere with a box
    around the body: the populations (the grid average and interpolation the
    control volume adds each coarse step included) and the per-block force
    partials at the FP32 floor of the reference build."""
    name = "geom_d3q19_cv"
    if not (GOLDEN / f"{name}.npz").exists():
        pytest.skip("control-volume fixture not generated")
    g = load(name)
    p, steps = geom_params(g)
    assert p.S_FORCE_TYPE == 1
    with ag.Case(p) as c:
        c.set_geometry(faces_of(g))
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(steps)
        c.sync()
        nmb, MC, Q = p.n_maxcblocks, int(g["MC"]), int(g["Q"])
        blocks = g["blocks"].astype(np.int64)
        fb = blocks[g["F_blocks"]] if "F_blocks" in g else blocks
        F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, fb, :].transpose(1, 0, 2)
        assert np.abs(F - g["F"][:, :Q, :].astype(np.float64)).max() < 2e-6
        Ff = c.dump(_lib.ARR_CBLOCK_F_FF).reshape(6, nmb)[:, blocks].T
        ref = g["Ff"].astype(np.float64)
        assert np.abs(ref).max() > 0
        assert np.abs(Ff - ref).max() < 5e-6 * np.abs(ref).max()
        # the FP64 report sums those partials (rows with surface terms cancel,
        # so the block-wise comparison above is the parity check) and resets them
        sums = c.forces()
        for r in range(6):
            assert abs(sums[r] - Ff[:, r].sum()) <= 1e-12 * (np.abs(Ff[:, r]).sum() + 1e-30)
        assert np.all(c.dump(_lib.ARR_CBLOCK_F_FF) == 0.0)


@pytest.mark.parametrize("mli", [2, 3])
def test_solution_refinement_with_geometry_fp64_matches_oracle(mli):
    """Near-wall refinement around the sphere, then the percentile rule every
    8 steps (grid average, interface interpolation, refine/coarsen pass with
    wall blocks present): meshes, masks and wall slots bit-exact and
    populations within 1e-11 of the FP64 oracle after four regrids."""
    from oracle.orc import OracleCase
    g = load("geom_d3q19_wall3_bouzidi")
    p, _ = geom_params(g)
    p.MAX_LEVELS_INTERIOR = mli
    p.S_CRITERION = _lib.CRITERION_PERCENTILE
    p.P_REFINE = 8
    p.ref_pct_hi = 0.5
    p.storage = _lib.STORE_FP64
    p.n_maxcblocks = max(p.n_maxcblocks, 4096)
    steps = 32
    runs = []
    for make in (lambda: ag.Case(p), lambda: OracleCase(p, p.n_maxcblocks, fp64=True)):
        c = make()
        c.set_geometry(faces_of(g))
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(steps)
        runs.append(c)
    c, o = runs
    c.sync()
    assert c.counts()["n_ids"] == o.counts()["n_ids"]
    for k in INT_ARRAYS:
        assert np.array_equal(c.dump(k), o.dump(k)), k
    nmb, Q, MC = p.n_maxcblocks, int(g["Q"]), int(g["MC"])
    ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    cnt = c.counts()
    blocks = np.sort(np.concatenate([ids[L, : cnt["n_ids"][L]] for L in range(cnt["max_levels"])])).astype(np.int64)
    Fc = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    Fo = o.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    assert np.abs(Fc - Fo).max() < 1e-11
    c.close()


@pytest.mark.parametrize("name", ["geom_d3q19_wall3_bouzidi", "geom_d3q27_wall2_bb"])
def test_wall_step_variants_and_graph_bit_identical(name):
    """Interpolated bounce-back (wall step) and plain bounce-back through the
    solid cells (the row variant's per-cell path next to solid cells)."""
    g = load(name)
    runs = []
    for variant, graph in [(1, True), (2, True), (3, True), (4, True), (5, True), (6, True), (1, False)]:
        c, p = run_case(g, variant=variant, use_graph=graph, steps=8)
        runs.append((c.dump(_lib.ARR_F), c.dump(_lib.ARR_CBLOCK_F_FF)))
        c.close()
    for F, Ff in runs[1:]:
        assert np.array_equal(F, runs[0][0])
        assert np.array_equal(Ff, runs[0][1])


def test_fp16_wall_flow_close_to_fp64():
    g = load("geom_d3q27_wall2_bb")
    c64, p = run_case(g, storage=_lib.STORE_FP64)
    c16, _ = run_case(g, storage=_lib.STORE_FP16)
    nmb, Q, MC = p.n_maxcblocks, int(g["Q"]), int(g["MC"])
    blocks = g["blocks"].astype(np.int64)
    F64 = c64.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    F16 = c16.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    solid = (c64.dump(_lib.ARR_CELLS_ID_MASK).reshape(nmb, MC)[blocks] == -1)[None]
    assert np.abs(np.where(solid, 0, F16 - F64)).max() < 2e-3
    f64, f16 = c64.forces(), c16.forces()
    assert abs(f16[0] - f64[0]) < 0.05 * abs(f64[0])
    c64.close()
    c16.close()


def test_geometry_refuses_2d_and_outside_faces():
    p = ag.default_params(velocity_set=_lib.D2Q9, Nx=32, n_maxcblocks=256)
    c = ag.Case(p)
    with pytest.raises(RuntimeError):
        c.set_geometry(np.zeros((1, 3, 3), np.float32))
    c.close()
    g = load("geom_d3q19_uniform")
    p, _ = geom_params(g)
    c = ag.Case(p)
    faces = faces_of(g).reshape(-1, 3, 3).copy()
    # A face across x = 0, met by a +x ray: its grown box reaches bins below x = 0.
    faces[0] = [[-0.02, 0.45, 0.45], [0.05, 0.6, 0.45], [0.0, 0.45, 0.6]]
    with pytest.raises(RuntimeError):
        c.set_geometry(faces)
    c.close()
