"""Parity of the CUDA multi-level path (interpolation, averaging, criterion,
refine/coarsen pass, S_Advance recursion) with the CPU oracle and with the
reference's own CUDA build.

Integer arrays (block IDs, neighbour and child lists, masks, ID sets, gap
stack, id_max) must be bit-exact.  Populations: FP64 storage against the FP64
oracle within 1e-12 (max abs; 1e-11 across refinement passes); FP32 against
the reference build within the floor-based bound of compare_to_golden; FP16
against FP64 within 1e-3 relative L2 of u."""
import numpy as np
import pytest

from helpers import lattice, macros_from_F, rel_l2
from test_oracle import (GOLDEN_CASES, REGRID_PAIRS, compare_to_golden, load_golden, params_for_golden,
                         regrid_from_reference, run_like_reference)

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu

AMR_CASES = [n for n in GOLDEN_CASES if n.startswith("amr_")]
INT_ARRAYS = (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_F_X, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR,
              _lib.ARR_CBLOCK_ID_NBR_CHILD, _lib.ARR_CBLOCK_ID_ONB, _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL)


def amr_params(Q=9, N=32, storage=_lib.STORE_FP64, **kw):
    dim = 2 if Q == 9 else 3
    vs = {9: _lib.D2Q9, 19: _lib.D3Q19, 27: _lib.D3Q27}[Q]
    base = dict(velocity_set=vs, Nx=N, v0=5e-5, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=3, P_REFINE=8,
                N_REFINE_START=-2.0, N_REFINE_INC=1.0, N_REFINE_MAX=1.0, storage=storage,
                bc_preset=_lib.BC_LDC2D if dim == 2 else _lib.BC_LDC3D,
                interp_order=_lib.INTERP_CUBIC if dim == 2 else _lib.INTERP_LINEAR)
    base.update(kw)
    ml = max(base["MAX_LEVELS_WALL"], base["MAX_LEVELS_INTERIOR"])
    n0 = (N // 4) ** dim
    base.setdefault("n_maxcblocks", sum(n0 * (4 if dim == 2 else 8) ** L for L in range(ml)) + 64)
    return ag.default_params(**base)


def compare_states(c, o, p, f_tol):
    """Product case c vs oracle case o: counts and integer arrays bit-exact,
    populations of the active blocks within f_tol (max abs)."""
    cc, oc = c.counts(), o.counts()
    assert cc["n_ids"] == oc["n_ids"] and cc["id_max"] == oc["id_max"] and cc["n_gaps"] == oc["n_gaps"]
    for k in INT_ARRAYS:
        assert (c.dump(k) == o.dump(k)).all(), k
    nmb = p.n_maxcblocks
    ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    ido = o.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    blocks = []
    for L in range(cc["max_levels"]):
        n = cc["n_ids"][L]
        assert (ids[L, :n] == ido[L, :n]).all(), L
        blocks.extend(ids[L, :n].tolist())
    n_gaps = cc["n_gaps"]
    assert (c.dump(_lib.ARR_GAP_SET)[:n_gaps] == o.dump(_lib.ARR_GAP_SET)[:n_gaps]).all()
    blocks = np.array(sorted(blocks), dtype=np.int64)
    Q, MC = c.Q, c.M_CBLOCK
    F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    Fo = o.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, blocks]
    err = np.abs(F - Fo).max()
    assert err < f_tol, err
    return err


@pytest.mark.parametrize("Q,N,kw", [
    (9, 32, dict(MAX_LEVELS_WALL=3, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOX)),
    (9, 32, dict(MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOUNDARY,
                 interp_order=_lib.INTERP_LINEAR)),
    (19, 16, dict(MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOX)),
    (27, 8, dict(MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOUNDARY,
                 interp_order=_lib.INTERP_CUBIC)),
])
def test_static_hierarchy_fp64_matches_oracle(Q, N, kw):
    """Near-wall / region refinement, then 40 coarse steps of the multi-level
    recursion (interpolation, per-level steps, averaging) in FP64."""
    from oracle.orc import OracleCase
    p = amr_params(Q, N, **kw)
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    run_like_reference(o, p, 40)
    with ag.Case(p) as c:
        run_like_reference(c, p, 40)
        c.sync()
        compare_states(c, o, p, 1e-12)


@pytest.mark.parametrize("Q,N,steps,kw", [
    (9, 32, 96, dict()),
    (9, 32, 96, dict(interp_order=_lib.INTERP_LINEAR, MAX_LEVELS_WALL=2, region_preset=_lib.REGION_BOUNDARY)),
    (19, 16, 24, dict(MAX_LEVELS_INTERIOR=2, v0=2.5e-5)),
])
def test_solution_refinement_fp64_matches_oracle(Q, N, steps, kw):
    """Solution-based refinement every P_REFINE coarse steps: criterion marks,
    refine/coarsen pass (ID recycling, neighbour rebuild) and the data moved
    into new children, against the FP64 oracle."""
    from oracle.orc import OracleCase
    p = amr_params(Q, N, **kw)
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    run_like_reference(o, p, steps)
    with ag.Case(p) as c:
        run_like_reference(c, p, steps)
        c.sync()
        assert c.refine_stats()["iter"] == steps
        compare_states(c, o, p, 1e-11)
        assert c.counts()["n_ids"][1] > 0


def test_transfers_fp64_match_oracle():
    """Each transfer alone on a refined state: interpolation into interface
    ghosts, averaging in every mode, and the criterion marks."""
    from oracle.orc import OracleCase
    p = amr_params(9, 32, MAX_LEVELS_WALL=3, MAX_LEVELS_INTERIOR=3, region_preset=_lib.REGION_BOX,
                   ic_preset=_lib.IC_UNIFORM, ic_noise=0.5, seed=11, u_ref=0.05)
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    o.set_ic(0)
    o.refine_near_wall()
    with ag.Case(p) as c:
        c.set_ic(0)
        c.refine_near_wall()
        compare_states(c, o, p, 1e-15)
        for L in (0, 1):
            c.interpolate(L, _lib.INTERP_INTERFACE)
            o.interpolate(L, _lib.INTERP_INTERFACE)
            compare_states(c, o, p, 1e-14)
        for var in (_lib.AVERAGE_INTERFACE, _lib.AVERAGE_BLOCK, _lib.AVERAGE_GRID):
            for L in (1, 0):
                c.average(L, var)
                o.average(L, var)
                compare_states(c, o, p, 1e-14)
        c.ref_criteria()
        o.ref_criteria()
        c.sync()
        assert (c.dump(_lib.ARR_CBLOCK_ID_REF) == o.dump(_lib.ARR_CBLOCK_ID_REF)).all()


@pytest.mark.parametrize("storage", [_lib.STORE_FP32, _lib.STORE_FP16])
def test_graph_replay_matches_eager(storage):
    """Captured coarse steps (two parities cached) give the same bits as eager
    launches, across refinement passes; after a regrid the captured step is
    updated in place rather than instantiated again."""
    p = amr_params(9, 32, storage=storage)
    res = []
    for graph in (False, True):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.refine_near_wall()
            c.advance_n(40, use_graph=graph)
            c.sync()
            res.append((c.dump(_lib.ARR_F), c.dump(_lib.ARR_ID_SET), c.counts()))
            if graph:
                gs = c.graph_stats()
                print(gs)
                assert gs["updates"] >= 1 and gs["builds"] >= 1, gs
    assert res[0][2] == res[1][2]
    assert (res[0][1] == res[1][1]).all()
    assert (res[0][0] == res[1][0]).all()


def test_fp16_multilevel_accuracy():
    """FP16 weight-offset storage through the multi-level recursion stays
    within 1e-3 relative L2 of u (1e-5 of rho) of the FP64 run on the same mesh."""
    kw = dict(MAX_LEVELS_WALL=3, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOX)
    out = {}
    for st in (_lib.STORE_FP64, _lib.STORE_FP16):
        p = amr_params(9, 32, storage=st, v0=5e-4, **kw)
        with ag.Case(p) as c:
            run_like_reference(c, p, 200)
            c.sync()
            out[st] = c.dump(_lib.ARR_F).reshape(9, p.n_maxcblocks, 16)
            ids = c.dump(_lib.ARR_ID_SET)
            cnt = c.counts()
    nmb = p.n_maxcblocks
    blocks = np.concatenate([ids.reshape(-1, nmb)[L, : cnt["n_ids"][L]] for L in range(3)])
    pb, cv, _ = lattice(9)
    r64, u64 = macros_from_F(out[_lib.STORE_FP64][:, blocks].reshape(9, -1), 2, 9, pb, cv)
    r16, u16 = macros_from_F(out[_lib.STORE_FP16][:, blocks].reshape(9, -1), 2, 9, pb, cv)
    assert rel_l2(np.stack(u16), np.stack(u64)) < 1e-3
    assert rel_l2(r16, r64) < 1e-5


@pytest.mark.skipif(not AMR_CASES, reason="no reference dumps committed")
@pytest.mark.parametrize("name", AMR_CASES)
def test_cuda_amr_vs_reference_build(name):
    g = load_golden(name)
    p, steps = params_for_golden(g)
    with ag.Case(p) as c:
        run_like_reference(c, p, steps)
        c.sync()
        compare_to_golden(g, c.dump, 1e-5, c.counts())


@pytest.mark.skipif(not REGRID_PAIRS, reason="no reference regrid dumps committed")
@pytest.mark.parametrize("name", REGRID_PAIRS)
def test_cuda_regrid_vs_reference_build(name):
    """The reference state before a refinement loaded into the CUDA library:
    criterion, marks and refine/coarsen pass give the reference's state after
    it bit for bit (integer arrays), on identical inputs."""
    c = regrid_from_reference(lambda p, nmb: ag.Case(ag.default_params(**{
        **{k: getattr(p, k) for k, _ in p._fields_}, "n_maxcblocks": nmb})), name)
    c.close()


ALL_ARRAYS = INT_ARRAYS + (_lib.ARR_ID_SET, _lib.ARR_GAP_SET, _lib.ARR_F)


@pytest.mark.parametrize("Q,N,storage,ml", [(9, 32, _lib.STORE_FP32, 3), (9, 32, _lib.STORE_FP64, 3),
                                            (19, 16, _lib.STORE_FP32, 3), (27, 16, _lib.STORE_FP64, 3),
                                            (9, 1032, _lib.STORE_FP32, 2)])
def test_percentile_marks_bit_exact_on_identical_inputs(Q, N, storage, ml):
    """The percentile criterion (block vorticity maxima, exact device
    quantile selection, marks) on the CUDA library and on the oracle, given
    the same populations and mesh: identical marks.  The 1032^2 case holds
    more than 65,536 blocks, so its quantiles come from the multi-CTA passes
    instead of the one-CTA selection."""
    from oracle.orc import OracleCase
    p = amr_params(Q, N, storage=storage, S_CRITERION=_lib.CRITERION_PERCENTILE, P_REFINE=8,
                   MAX_LEVELS_INTERIOR=ml, v0=5e-4)
    with ag.Case(p) as c:
        run_like_reference(c, p, 12)   # one regrid done, the hierarchy still growing
        c.sync()
        o = OracleCase(p, p.n_maxcblocks, fp64=(storage == _lib.STORE_FP64))
        for k in ALL_ARRAYS:
            o.load(k, c.dump(k))
        cnt = c.counts()
        o.set_counts(cnt["n_ids"], cnt["id_max"], cnt["n_gaps"])
        assert cnt["n_ids"][1] > 0
        for L in range(cnt["max_levels"]):
            c.refresh(L)
            o.refresh(L)
        c.ref_criteria()
        o.ref_criteria()
        c.sync()
        r, ro = c.dump(_lib.ARR_CBLOCK_ID_REF), o.dump(_lib.ARR_CBLOCK_ID_REF)
        assert (r == ro).all()
        assert ((r == 4) | (r == 5)).any()   # marks to refine (4) or coarsen (5) exist


@pytest.mark.parametrize("Q,N,steps", [(9, 32, 96), (19, 16, 32)])
def test_percentile_refinement_fp64_matches_oracle(Q, N, steps):
    """Percentile-driven refinement every P_REFINE coarse steps in FP64:
    meshes bit-exact and populations within 1e-11 of the FP64 oracle."""
    from oracle.orc import OracleCase
    p = amr_params(Q, N, S_CRITERION=_lib.CRITERION_PERCENTILE, MAX_LEVELS_INTERIOR=3 if Q == 9 else 2,
                   v0=5e-4 if Q == 9 else 2.5e-4)
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    run_like_reference(o, p, steps)
    with ag.Case(p) as c:
        run_like_reference(c, p, steps)
        c.sync()
        compare_states(c, o, p, 1e-11)


def test_nearly_full_pool_matches_oracle():
    """A block pool of 175 on a 64-block root grid with three levels: at some
    regrid the blocks marked for refinement fit the gap stack although
    id_max + 4 x marks passes the pool size (mesh_amr.cu:2186).  Every pass
    stops at the pool size; mesh bit-exact, populations within 1e-11 of the
    FP64 oracle through the regrids that follow."""
    from oracle.orc import OracleCase
    nmb, P = 175, 8
    p = amr_params(9, 32, n_maxcblocks=nmb, P_REFINE=10 ** 8, S_CRITERION=_lib.CRITERION_PERCENTILE,
                   ref_pct_hi=0.8, ref_pct_lo=0.5, v0=5e-4)
    o = OracleCase(p, nmb, fp64=True)
    hit = False
    with ag.Case(p) as c:
        for case in (c, o):
            case.set_ic(0)
        for _ in range(16):
            for case in (c, o):
                case.advance_n(P)
                for L in (1, 0):
                    case.average(L, _lib.AVERAGE_GRID)
                for L in (0, 1):
                    case.interpolate(L, _lib.INTERP_INTERFACE)
                case.ref_criteria()
            cnt = o.counts()
            n_r = int((o.dump(_lib.ARR_CBLOCK_ID_REF) == 4).sum())
            hit |= 0 < 4 * n_r <= cnt["n_gaps"] and cnt["id_max"][3] + 4 * n_r > nmb
            for case in (c, o):
                case.refine_coarsen()
        c.sync()
        assert hit
        compare_states(c, o, p, 1e-11)


@pytest.mark.parametrize("Q,N,storage,kw", [
    (9, 32, _lib.STORE_FP16, dict(MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=3, S_CRITERION=_lib.CRITERION_PERCENTILE)),
    (9, 32, _lib.STORE_FP32, dict(MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=3, region_preset=_lib.REGION_BOUNDARY)),
    (19, 16, _lib.STORE_FP16, dict(MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=1, region_preset=_lib.REGION_BOX)),
    (27, 8, _lib.STORE_BF16, dict(MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=2, S_CRITERION=_lib.CRITERION_PERCENTILE)),
])
def test_row_variant_bit_identical_on_multilevel_runs(Q, N, storage, kw):
    """The row-mapped step (variant 4) through interface blocks with missing
    same-level neighbours, the boundary hook and regrids, and the root-level
    tile steps (variants 5 and 6, 2D): the same populations and mesh as one
    cell per thread, bit for bit."""
    p = amr_params(Q, N, storage=storage, **kw)
    out = []
    for v in (1, 4, 5, 6):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.set_tuning(v)
            c.refine_near_wall()
            c.advance_n(48, use_graph=True)
            c.sync()
            out.append((c.dump(_lib.ARR_F), c.dump(_lib.ARR_ID_SET), c.counts()["n_ids"]))
    assert max(out[0][2][1:]) > 0
    for o in out[1:]:
        assert out[0][2] == o[2]
        assert np.array_equal(out[0][1], o[1])
        assert np.array_equal(out[0][0], o[0])
