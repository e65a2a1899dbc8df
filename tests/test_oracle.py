"""The CPU oracle against the reference: lattice tables and root grid
bit-exact against the golden vectors extracted from the reference sources,
and populations against the reference's own CUDA build (golden dumps in
tests/golden/*.npz, made by tests/golden/make_golden.py on a B200)."""
import json

import numpy as np
import pytest

from helpers import GOLDEN, brute_root_grid, lattice, macros_from_F, rel_l2, tables

import agal_b200 as ag
from agal_b200 import _lib


def test_golden_tables_consistent():
    t = tables()
    # D3Q19 is the first 19 directions of the D3Q27 order; opposites are involutions.
    for key in ["LBMpb_D2Q9", "LBMpb_D3Q19", "LBMpb_D3Q27"]:
        pb = t[key]
        assert all(pb[pb[p]] == p for p in range(len(pb)))
    c = np.array(t["V_CONN_ID_3D"]).reshape(3, 27)
    for p, q in enumerate(t["LBMpb_D3Q27"]):
        assert (c[:, p] == -c[:, q]).all()
    assert abs(sum(t["LBMw_D2Q9"]) - 1) < 1e-15 and abs(sum(t["LBMw_D3Q27"]) - 1) < 1e-15
    # block-neighbour directions of mesh.h equal the D2Q9 / D3Q27 velocities
    assert t["MESH_C_3D"] == t["V_CONN_ID_3D"]
    assert t["MESH_C_2D"] == t["V_CONN_ID_2D"][:9] + t["V_CONN_ID_2D"][27:36]


@pytest.mark.parametrize("vs,N,per", [(0, (32, 32, 1), (0, 0, 0)), (0, (32, 16, 1), (1, 0, 0)),
                                      (0, (16, 32, 1), (0, 1, 0)), (1, (16, 16, 16), (0, 0, 0)),
                                      (2, (16, 8, 12), (1, 0, 1)), (1, (8, 16, 8), (0, 1, 1))])
def test_oracle_root_grid_bit_exact(oracle_lib, vs, N, per):
    from oracle.orc import OracleCase
    Nx, Ny, Nz = N
    p = ag.default_params(velocity_set=vs, Nx=Nx, L_fy=Ny / Nx, L_fz=Nz / Nx, MAX_LEVELS_WALL=1,
                          MAX_LEVELS_INTERIOR=1, PERIODIC_X=per[0], PERIODIC_Y=per[1], PERIODIC_Z=per[2])
    dim = 2 if vs == 0 else 3
    nb_exp, onb_exp = brute_root_grid(dim, Nx, Ny, Nz, per)
    n = nb_exp.shape[1]
    nmb = n + 37
    o = OracleCase(p, nmb)
    Qmax = 9 if dim == 2 else 27
    nbr = o.dump(_lib.ARR_CBLOCK_ID_NBR).reshape(Qmax, nmb)
    assert (nbr[:, :n] == nb_exp).all()
    assert (nbr[:, n:] == -999).all()
    onb = o.dump(_lib.ARR_CBLOCK_ID_ONB)
    assert (onb[:n] == onb_exp).all()
    ch = o.dump(_lib.ARR_CBLOCK_ID_NBR_CHILD).reshape(Qmax, nmb)
    assert (ch[:, :n] == np.where(nb_exp < 0, nb_exp, -999)).all()
    gaps = o.dump(_lib.ARR_GAP_SET)
    assert (gaps[: nmb - n] == np.arange(nmb - 1, n - 1, -1)).all()
    ids = o.dump(_lib.ARR_ID_SET)
    assert (ids[:n] == np.arange(n)).all()
    c = o.counts()
    assert c["n_ids"][0] == n and c["n_gaps"] == nmb - n and c["id_max"][0] == n


def test_oracle_rest_state_is_fixed_point(oracle_lib):
    from oracle.orc import OracleCase
    p = ag.default_params(velocity_set=_lib.D3Q19, Nx=8, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=1e-3)
    o = OracleCase(p, 8, fp64=True)
    o.set_ic(0)
    f0 = o.dump(_lib.ARR_F)
    o.advance_n(20)
    assert np.abs(o.dump(_lib.ARR_F) - f0).max() < 1e-15


def test_oracle_periodic_mass_momentum_conserved(oracle_lib):
    from oracle.orc import OracleCase
    p = ag.default_params(velocity_set=_lib.D2Q9, Nx=32, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=1e-3,
                          PERIODIC_X=1, PERIODIC_Y=1, ic_preset=_lib.IC_UNIFORM, ic_noise=0.2, seed=7)
    o = OracleCase(p, 64, fp64=True)
    o.set_ic(0)
    m0 = o.mass_momentum()
    o.advance_n(50)
    m1 = o.mass_momentum()
    assert abs(m1[0] - m0[0]) < 1e-10 * m0[0]
    assert np.abs(m1[1:] - m0[1:]).max() < 1e-10 * m0[0]


# ---------------------------------------------------------------------------
# Against the reference's own CUDA build (fixtures from a B200 run).
GOLDEN_CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    d = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    return {k: d[k] for k in d.files}


def params_for_golden(g):
    keys = json.loads(str(g["case_keys"]))
    vs = {9: _lib.D2Q9, 19: _lib.D3Q19, 27: _lib.D3Q27}[int(g["Q"])]
    bc = _lib.BC_LDC2D if int(g["dim"]) == 2 else _lib.BC_LDC3D
    # Block IDs are taken from the low end of the gap stack (the stack holds
    # n_maxcblocks-1 .. n_coarse, popped from the end), so they do not depend
    # on the pool size: a pool just above the largest active ID reproduces the
    # reference's IDs without its multi-GB allocation.
    # A multi-level case can hold more IDs in passing than at the end, so its
    # pool covers the fully refined hierarchy.
    ml = int(g["max_levels"])
    nch = 4 if int(g["dim"]) == 2 else 8
    n0 = int(g["n_ids"][0]) if ml == 1 else int(np.sum(g["level"][:, 0] == 0))
    full = sum(n0 * nch ** L for L in range(ml))
    nmb = max(int(g["blocks"].max()) + 1, full if ml > 1 else 0) + 64
    interp = _lib.INTERP_LINEAR if (int(g["dim"]) == 3 or str(g["binary"]).endswith("_lin")) else _lib.INTERP_CUBIC
    region = int(g["region"]) if "region" in g else 0
    kw = dict(velocity_set=vs, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, bc_preset=bc,
              ic_preset=_lib.IC_REST, n_maxcblocks=nmb, interp_order=interp, region_preset=region)
    kw.update(keys)
    return ag.default_params(**kw), int(g["steps"])


def run_like_reference(case, p, steps):
    """The reference driver's sequence: IC, near-wall refinement when the
    hierarchy has more than one level, then the M_AdvanceLoop body."""
    case.set_ic(0)
    if max(p.MAX_LEVELS_WALL, p.MAX_LEVELS_INTERIOR) > 1:
        case.refine_near_wall()
    case.advance_n(steps)


def fp64_floor(g):
    """rho/u of an FP64 oracle run of the golden case, and the distance of the
    reference's own FP32 result from it (its FP32 round-off floor)."""
    from oracle.orc import OracleCase
    p, steps = params_for_golden(g)
    Q, dim, MC = int(g["Q"]), int(g["dim"]), int(g["MC"])
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    run_like_reference(o, p, steps)
    blocks = g["blocks"].astype(np.int64)
    F = o.dump(_lib.ARR_F).reshape(Q, p.n_maxcblocks, MC)[:, blocks, :].reshape(Q, -1)
    pb, c, _ = lattice(Q)
    rho64, u64 = macros_from_F(F, dim, Q, pb, c)
    Fr = np.transpose(g["F"][:, :Q, :], (1, 0, 2)).reshape(Q, -1).astype(np.float64)
    rho_r, u_r = macros_from_F(Fr, dim, Q, pb, c)
    return rho64, np.stack(u64), rel_l2(np.stack(u_r), np.stack(u64)), rel_l2(rho_r, rho64)


def compare_ints(g, dumpf, counts=None):
    """Block and cell integer arrays of the dump's active blocks, the ID sets,
    and (with counts) n_ids, id_max and the top of the gap stack: bit-exact."""
    blocks = g["blocks"].astype(np.int64)
    dim, Qmax, MC = int(g["dim"]), int(g["Qmax"]), int(g["MC"])
    nmb = len(dumpf(_lib.ARR_CBLOCK_ID_ONB))
    if counts is not None:
        ml = int(g["max_levels"])
        assert counts["n_ids"][:ml] == [int(v) for v in g["n_ids"][:ml]]
        assert counts["id_max"][: ml + 1] == [int(v) for v in g["id_max"][: ml + 1]]
        gaps = dumpf(_lib.ARR_GAP_SET)[: counts["n_gaps"]]
        tail = g["gaps_tail"]
        k = 0
        while k < min(len(tail), len(gaps)) and tail[len(tail) - 1 - k] < nmb - 64:
            k += 1
        assert (gaps[len(gaps) - k:] == tail[len(tail) - k:]).all()
    assert (dumpf(_lib.ARR_CBLOCK_ID_NBR).reshape(Qmax, nmb)[:, blocks].T == g["nbr"]).all()
    assert (dumpf(_lib.ARR_CBLOCK_ID_NBR_CHILD).reshape(Qmax, nmb)[:, blocks].T == g["nbr_child"]).all()
    for arr, key in [(_lib.ARR_CBLOCK_ID_ONB, "onb"), (_lib.ARR_CBLOCK_ID_REF, "ref"),
                     (_lib.ARR_CBLOCK_LEVEL, "level"), (_lib.ARR_CBLOCK_ID_MASK, "bmask")]:
        assert (dumpf(arr)[blocks] == g[key][:, 0]).all(), key
    assert (dumpf(_lib.ARR_CBLOCK_F_X).reshape(dim, nmb)[:, blocks].T == g["fX"]).all()
    assert (dumpf(_lib.ARR_CELLS_ID_MASK).reshape(nmb, MC)[blocks] == g["cmask"]).all()
    for L in range(int(g["max_levels"])):
        n = int(g["n_ids"][L])
        assert (dumpf(_lib.ARR_ID_SET).reshape(-1, nmb)[L, :n] == g[f"id_set_{L}"]).all()


def load_reference_state(case, g, nmb):
    """Load a reference dump (its active blocks) into an nmb-block pool of the
    oracle or the CUDA library, with the counts of the restart reader.  Blocks
    outside the dump take a fresh pool's values; the gap stack keeps the
    dump's top (recycled and lowest fresh IDs, in stack order) over the
    remaining free IDs of the smaller pool, in descending order."""
    dim, Q, Qmax, MC, ML = (int(g[k]) for k in ("dim", "Q", "Qmax", "MC", "max_levels"))
    blocks = g["blocks"].astype(np.int64)
    cm = np.zeros((nmb, MC), np.int32)
    cm[blocks] = g["cmask"]
    fX = np.zeros((dim, nmb), np.float32)
    fX[:, blocks] = g["fX"].T
    arrs = {_lib.ARR_CELLS_ID_MASK: cm, _lib.ARR_CBLOCK_F_X: fX}
    for arr, key, fill in [(_lib.ARR_CBLOCK_ID_MASK, "bmask", 0), (_lib.ARR_CBLOCK_ID_ONB, "onb", 0),
                           (_lib.ARR_CBLOCK_ID_REF, "ref", 8), (_lib.ARR_CBLOCK_LEVEL, "level", 0)]:
        a = np.full(nmb, fill, np.int32)
        a[blocks] = g[key][:, 0]
        arrs[arr] = a
    for arr, key in [(_lib.ARR_CBLOCK_ID_NBR, "nbr"), (_lib.ARR_CBLOCK_ID_NBR_CHILD, "nbr_child")]:
        a = np.full((Qmax, nmb), -999, np.int32)
        a[:, blocks] = g[key].T
        arrs[arr] = a
    ids = np.zeros((ML, nmb), np.int32)
    for L in range(ML):
        v = g[f"id_set_{L}"]
        ids[L, : len(v)] = v
    arrs[_lib.ARR_ID_SET] = ids
    tail = g["gaps_tail"]
    top = []
    for v in tail[::-1]:
        if v >= nmb:
            break
        top.append(int(v))
    top = top[::-1]
    used = set(top) | set(blocks.tolist())
    stack = [b for b in range(nmb - 1, -1, -1) if b not in used] + top
    gaps = np.zeros(nmb, np.int32)
    gaps[: len(stack)] = stack
    arrs[_lib.ARR_GAP_SET] = gaps
    F = np.zeros((Q, nmb * MC))
    Fr = F.reshape(Q, nmb, MC)
    Fr[:, blocks, :] = np.transpose(g["F"][:, :Q, :], (1, 0, 2))
    arrs[_lib.ARR_F] = F
    for k, a in arrs.items():
        case.load(k, a.reshape(-1))
    case.set_counts([int(v) for v in g["n_ids"]], [int(v) for v in g["id_max"]], len(stack))


def compare_to_golden(g, dumpf, tol_rel_l2, counts=None):
    """Integer arrays bit-exact; rho/u against the reference's own FP32 build.

    Two FP32 implementations that round differently cannot agree to better
    than their round-off: the reference's FP32 result is itself 2e-5..8e-5
    (u, relative L2) away from an FP64 run of the same algorithm after
    100-1000 steps.  So rho and u must be within max(tol_rel_l2, 2 x that
    floor) of the reference, and no further from the FP64 result than
    1.5 x the reference's own distance."""
    blocks = g["blocks"].astype(np.int64)
    dim, Q, MC = int(g["dim"]), int(g["Q"]), int(g["MC"])
    nmb = len(dumpf(_lib.ARR_CBLOCK_ID_ONB))
    compare_ints(g, dumpf, counts)
    F = dumpf(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks, :].reshape(Q, -1)
    Fr = np.transpose(g["F"][:, :Q, :], (1, 0, 2)).reshape(Q, -1).astype(np.float64)
    pb, c, _ = lattice(Q)
    rho, u = macros_from_F(F, dim, Q, pb, c)
    rho_r, u_r = macros_from_F(Fr, dim, Q, pb, c)
    u, u_r = np.stack(u), np.stack(u_r)
    rho64, u64, floor_u, floor_rho = fp64_floor(g)
    assert rel_l2(rho, rho_r) < max(tol_rel_l2, 2 * floor_rho)
    assert rel_l2(u, u_r) < max(tol_rel_l2, 2 * floor_u), (rel_l2(u, u_r), floor_u)
    assert rel_l2(u, u64) <= 1.5 * floor_u + 1e-7, (rel_l2(u, u64), floor_u)
    assert rel_l2(rho, rho64) <= 1.5 * floor_rho + 1e-9
    return rel_l2(F, Fr)


REGRID_PAIRS = sorted(p.stem[: -len("_pre")] for p in GOLDEN.glob("regrid_*_pre.npz"))


def regrid_from_reference(case_factory, name):
    """Load the reference state before a refinement, refine, and compare with
    the reference state after it: integer arrays bit-exact, populations (the
    grid average and the data interpolated into new children) within 1e-6
    (linear interpolation) or 1e-4 (cubic).  The cubic bound is the
    reference's own rounding: it evaluates the interpolant in FP32 from
    monomial coefficients up to ~500 (util_interp.h), whose cancellation
    leaves 1e-5..1e-4 absolute error; the oracle and the CUDA library
    evaluate the same interpolant in the Lagrange form."""
    pre, post = load_golden(name + "_pre"), load_golden(name + "_post")
    p, _ = params_for_golden(post)
    nmb = p.n_maxcblocks
    case = case_factory(p, nmb)
    load_reference_state(case, pre, nmb)
    case.refine_with_solution()
    counts = case.counts()
    compare_ints(post, case.dump, counts)
    blocks = post["blocks"].astype(np.int64)
    Q, MC = int(post["Q"]), int(post["MC"])
    F = case.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks, :]
    Fr = np.transpose(post["F"][:, :Q, :], (1, 0, 2)).astype(np.float64)
    tol = 1e-4 if p.interp_order == _lib.INTERP_CUBIC else 1e-6
    assert np.abs(F - Fr).max() < tol
    return case


@pytest.mark.skipif(not REGRID_PAIRS, reason="no reference regrid dumps committed")
@pytest.mark.parametrize("name", REGRID_PAIRS)
def test_oracle_regrid_vs_reference_build(oracle_lib, name):
    from oracle.orc import OracleCase
    regrid_from_reference(lambda p, nmb: OracleCase(p, nmb), name)


GOLDEN_RUNS = [n for n in GOLDEN_CASES if not n.startswith(("regrid_", "geom_", "restart_", "faces_", "les_"))]


@pytest.mark.skipif(not GOLDEN_RUNS, reason="no reference dumps committed")
@pytest.mark.parametrize("name", GOLDEN_RUNS)
def test_oracle_vs_reference_build(oracle_lib, name):
    from oracle.orc import OracleCase
    g = load_golden(name)
    p, steps = params_for_golden(g)
    o = OracleCase(p, p.n_maxcblocks)
    run_like_reference(o, p, steps)
    compare_to_golden(g, o.dump, 1e-5, o.counts())


def test_oracle_percentile_criterion_refines_the_top_decile(oracle_lib):
    """Percentile mode: after the first regrid about a tenth of the leaf
    blocks (those above the 0.9 quantile of vorticity) are refined."""
    from oracle.orc import OracleCase
    p = ag.default_params(Nx=64, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=2, P_REFINE=16, v0=5e-5,
                          bc_preset=_lib.BC_LDC2D, S_CRITERION=_lib.CRITERION_PERCENTILE)
    o = OracleCase(p, 256 * 5 + 64)
    o.set_ic(0)
    o.advance_n(16)
    n1 = o.counts()["n_ids"][1]
    assert n1 % 4 == 0 and 0 < n1 // 4 <= 26   # floor(0.9 * 255) = 229: 26 blocks strictly above


def test_oracle_mrt_with_all_rates_omega_is_bgk(oracle_lib):
    """The D3Q19 MRT moment basis, its inverse and the legacy equilibria are
    consistent: with every rate equal to omega the collision is BGK."""
    from oracle.orc import OracleCase
    base = dict(velocity_set=_lib.D3Q19, Nx=8, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=1.25e-4,
                bc_preset=_lib.BC_LDC3D)
    om = (1.0 / 8) / (1.25e-4 * 3 + 0.5 / 8)
    a = OracleCase(ag.default_params(**base), 10, fp64=True)
    b = OracleCase(ag.default_params(**base, collision=_lib.MRT, s1=om, s2=om, s3=om, s5=om, s6=om), 10, fp64=True)
    for o in (a, b):
        o.set_ic(0)
        o.advance_n(30)
    assert np.abs(a.dump(_lib.ARR_F) - b.dump(_lib.ARR_F)).max() < 1e-13
