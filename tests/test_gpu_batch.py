"""Batched execution: cases advanced together in one graph per coarse step
(agal_batch_*) end bit for bit where advancing each alone leaves them,
regrids, walls and forces included."""
import numpy as np
import pytest

import agal_b200 as ag
from agal_b200 import _lib
from agal_b200.geometry import icosphere

pytestmark = pytest.mark.gpu


def case_specs():
    """A mixed batch: 2D multi-level with percentile regrids, 3D uniform
    cavity, 3D flow past a sphere with walls and forces, 2D FP16 uniform."""
    amr2d = dict(velocity_set=_lib.D2Q9, Nx=32, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=3, v0=5e-4, P_REFINE=8,
                 S_CRITERION=_lib.CRITERION_PERCENTILE, bc_preset=_lib.BC_LDC2D, storage=_lib.STORE_FP64,
                 n_maxcblocks=64 * 21 + 64)
    ldc3d = dict(velocity_set=_lib.D3Q19, Nx=16, v0=1.25e-4, bc_preset=_lib.BC_LDC3D, storage=_lib.STORE_FP32,
                 n_maxcblocks=80)
    geo3d = dict(velocity_set=_lib.D3Q27, Nx=16, MAX_LEVELS_WALL=2, MAX_LEVELS_INTERIOR=2, v0=1.25e-4,
                 P_REFINE=100000, G_BIN_DENSITY=8, G_BIN_LEVELS=2, G_BIN_SPEC=2, G_BIN_MAKE_LINKS=1,
                 G_NEAR_WALL_DISTANCE=0.05, S_BC_TYPE=1, S_FORCE_TYPE=0, S_FORCE_ORDER=2, bc_preset=_lib.BC_FPSC3D,
                 ic_preset=_lib.IC_UNIFORM, u_ref=0.05, storage=_lib.STORE_FP64, n_maxcblocks=64 * 9 + 64)
    ldc2d16 = dict(velocity_set=_lib.D2Q9, Nx=64, v0=5e-4, bc_preset=_lib.BC_LDC2D, storage=_lib.STORE_FP16,
                   n_maxcblocks=300)
    return [amr2d, ldc3d, geo3d, ldc2d16]


def make(spec):
    c = ag.Case(ag.default_params(**spec))
    if spec.get("S_FORCE_TYPE") == 0:
        c.set_geometry(icosphere(2, 0.12, (0.46, 0.5, 0.52), seed=5))
    c.set_ic(0)
    c.refine_near_wall()
    return c


def state(c):
    out = {k: c.dump(k) for k in (_lib.ARR_F, _lib.ARR_ID_SET, _lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_ID_NBR)}
    out["counts"] = c.counts()
    if c.params.S_FORCE_TYPE == 0 and c.params.S_BC_TYPE:
        out["Ff"] = c.dump(_lib.ARR_CBLOCK_F_FF)
    return out


@pytest.mark.parametrize("worklist", [True, False])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_equals_cases_alone(use_graph, worklist):
    steps = 20
    alone = []
    for spec in case_specs():
        c = make(spec)
        c.advance_n(steps)
        c.sync()
        alone.append(state(c))
        c.close()
    cases = [make(spec) for spec in case_specs()]
    with ag.Batch(cases) as b:
        b.set_worklist(worklist)
        b.advance_n(7, use_graph=use_graph)
        b.advance_n(steps - 7, use_graph=use_graph)
        b.sync()
    for i, c in enumerate(cases):
        s = state(c)
        assert s["counts"] == alone[i]["counts"], i
        for k in s:
            if k != "counts":
                assert np.array_equal(s[k], alone[i][k]), (i, k)
        c.close()
    # the multi-level case really regridded inside the batch
    assert alone[0]["counts"]["n_ids"][1] > 0


@pytest.mark.parametrize("worklist", [True, False])
def test_learned_cases_in_a_batch_equal_alone(worklist):
    """Cases driven by the learned predictor (look-ahead over 2 regrids, the
    rule judging every other regrid), each with its own network of the same
    weights, regrid inside a batch exactly as alone."""
    spec = dict(case_specs()[0], P_REFINE=4)
    specs = [dict(spec, v0=5e-4), dict(spec, v0=2.5e-4, Nx=48, n_maxcblocks=144 * 21 + 64)]
    steps = 24

    def learned(sp):
        c = make(sp)
        m = ag.Learner(2, seed=11)
        m.set_horizon(2)
        m.attach(c, 2, judge_every=2)
        m.set_thresholds(0.5, 0.5)
        return c, m

    alone = []
    for sp in specs:
        c, m = learned(sp)
        c.advance_n(steps)
        c.sync()
        alone.append(state(c))
        c.close()
        m.close()
    pairs = [learned(sp) for sp in specs]
    with ag.Batch([c for c, _ in pairs]) as b:
        b.set_worklist(worklist)
        b.advance_n(steps)
        b.sync()
    for i, (c, m) in enumerate(pairs):
        s = state(c)
        assert s["counts"] == alone[i]["counts"], i
        for k in s:
            if k != "counts":
                assert np.array_equal(s[k], alone[i][k]), (i, k)
        c.close()
        m.close()


def test_batch_rejects_duplicates():
    c = make(case_specs()[1])
    with pytest.raises(RuntimeError):
        ag.Batch([c, c])
    c.close()


def test_worklist_many_cases_of_one_kernel():
    """Work-list mode with several cases on one batched kernel: D2Q9 FP16
    cavities of different sizes and level counts (regrids every 8 steps), so
    each step phase holds cases with different chunk counts and some phases
    only part of the cases; every case ends bit for bit where it ends alone."""
    specs = []
    for k, (N, ml) in enumerate([(32, 3), (64, 1), (48, 2), (32, 2), (64, 3), (16, 1)]):
        specs.append(dict(velocity_set=_lib.D2Q9, Nx=N, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=ml, v0=5e-4 * (k + 1),
                          P_REFINE=8, S_CRITERION=_lib.CRITERION_PERCENTILE, bc_preset=_lib.BC_LDC2D,
                          storage=_lib.STORE_FP16, n_maxcblocks=(N // 4) ** 2 * 21 + 64))
    steps = 24
    alone = []
    for spec in specs:
        c = make(spec)
        c.advance_n(steps)
        c.sync()
        alone.append(state(c))
        c.close()
    cases = [make(spec) for spec in specs]
    with ag.Batch(cases) as b:
        b.set_worklist(True)
        b.advance_n(steps)
        b.sync()
    for i, c in enumerate(cases):
        s = state(c)
        assert s["counts"] == alone[i]["counts"], i
        for k in s:
            if k != "counts":
                assert np.array_equal(s[k], alone[i][k]), (i, k)
        c.close()


def test_batch_autotune_picks_a_mode_and_keeps_results():
    """The launch-mode autotuner times both modes on real steps: the cases
    advance 2 x (steps + 2) coarse steps and end where advancing them alone
    leaves them."""
    steps = 3
    total = 2 * (steps + 2) + 5
    alone = []
    for spec in case_specs():
        c = make(spec)
        c.advance_n(total)
        c.sync()
        alone.append(state(c))
        c.close()
    cases = [make(spec) for spec in case_specs()]
    with ag.Batch(cases) as b:
        r = b.autotune(steps)
        assert r["ms_branches"] > 0 and r["ms_worklist"] > 0
        b.advance_n(5)
        b.sync()
    for i, c in enumerate(cases):
        s = state(c)
        assert s["counts"] == alone[i]["counts"], i
        for k in s:
            if k != "counts":
                assert np.array_equal(s[k], alone[i][k]), (i, k)
        c.close()
