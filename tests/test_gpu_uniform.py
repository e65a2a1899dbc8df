"""Parity of the CUDA single-level step (fused collide + boundary + stream)
with the CPU oracle and with the reference's own CUDA build.

Tolerances: FP32 and FP64 storage compare the full population arrays;
rho and u are held to 1e-5 relative L2 (FP32) as the reference-parity bar.
FP16/BF16 weight-offset storage is compared with an FP64 oracle run:
relative L2 of u below 1e-3 (BF16: 1e-2), of rho below 1e-5 (BF16: 1e-4).
Integer arrays (root grid, masks, ID sets) must be bit-exact."""
import numpy as np
import pytest

from helpers import brute_root_grid, lattice, macros_from_F, rel_l2
from test_oracle import GOLDEN_CASES, compare_to_golden, load_golden, params_for_golden

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu

VS = {9: _lib.D2Q9, 19: _lib.D3Q19, 27: _lib.D3Q27}


def ldc_params(Q, N, steps_re=100.0, storage=_lib.STORE_FP32, extra=None):
    dim = 2 if Q == 9 else 3
    kw = dict(velocity_set=VS[Q], Nx=N, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=0.05 / steps_re,
              bc_preset=_lib.BC_LDC2D if dim == 2 else _lib.BC_LDC3D, storage=storage,
              n_maxcblocks=(N // 4) ** dim + 5)
    if extra:
        kw.update(extra)
    return ag.default_params(**kw)


def run_pair(p, steps, fp64_oracle=False, use_graph=False):
    from oracle.orc import OracleCase
    o = OracleCase(p, p.n_maxcblocks, fp64=fp64_oracle)
    o.set_ic(0)
    o.advance_n(steps)
    with ag.Case(p) as c:
        c.set_ic(0)
        if use_graph:
            c.advance_n(steps, use_graph=True)
        else:
            for _ in range(steps):
                c.advance()
        c.sync()
        F = c.dump(_lib.ARR_F)
        ints = {k: c.dump(k) for k in (_lib.ARR_CBLOCK_ID_NBR, _lib.ARR_CBLOCK_ID_NBR_CHILD, _lib.ARR_CBLOCK_ID_ONB,
                                       _lib.ARR_ID_SET, _lib.ARR_GAP_SET, _lib.ARR_CBLOCK_F_X)}
    oints = {k: o.dump(k) for k in ints}
    return F, o.dump(_lib.ARR_F), ints, oints


def active(F, Q, nmb, n):
    MC = F.size // (Q * nmb)
    return F.reshape(Q, nmb, MC)[:, :n, :].reshape(Q, -1)


@pytest.mark.parametrize("Q,N,steps", [(9, 64, 500), (9, 128, 200), (19, 16, 100), (27, 16, 100), (19, 32, 50)])
def test_fp32_step_matches_oracle(Q, N, steps):
    """FP32 CUDA vs FP32 oracle.  The two round differently (the GPU build
    fuses multiply-adds, the oracle is compiled without contraction), so after
    hundreds of steps u differs at the 1e-5 level; the test therefore also
    requires the CUDA result to be as close to an FP64 oracle run as the FP32
    oracle itself is."""
    from oracle.orc import OracleCase
    p = ldc_params(Q, N)
    F, Fo, ints, oints = run_pair(p, steps)
    for k in ints:
        assert (ints[k] == oints[k]).all(), k
    dim = 2 if Q == 9 else 3
    n = (N // 4) ** dim
    A, B = active(F, Q, p.n_maxcblocks, n), active(Fo, Q, p.n_maxcblocks, n)
    pb, c, _ = lattice(Q)
    rho, u = macros_from_F(A, dim, Q, pb, c)
    rho_o, u_o = macros_from_F(B, dim, Q, pb, c)
    assert rel_l2(rho, rho_o) < 1e-5
    assert rel_l2(np.stack(u), np.stack(u_o)) < 5e-5
    assert np.abs(A - B).max() < 1e-5
    o64 = OracleCase(p, p.n_maxcblocks, fp64=True)
    o64.set_ic(0)
    o64.advance_n(steps)
    rho_d, u_d = macros_from_F(active(o64.dump(_lib.ARR_F), Q, p.n_maxcblocks, n), dim, Q, pb, c)
    e_cuda = rel_l2(np.stack(u), np.stack(u_d))
    e_orc = rel_l2(np.stack(u_o), np.stack(u_d))
    assert e_cuda <= 2.0 * e_orc + 1e-7, (e_cuda, e_orc)


@pytest.mark.parametrize("Q", [9, 19, 27])
def test_fp64_step_matches_fp64_oracle(Q):
    N = 32 if Q == 9 else 12
    p = ldc_params(Q, N, storage=_lib.STORE_FP64)
    F, Fo, _, _ = run_pair(p, 100, fp64_oracle=True)
    dim = 2 if Q == 9 else 3
    n = (N // 4) ** dim
    assert np.abs(active(F, Q, p.n_maxcblocks, n) - active(Fo, Q, p.n_maxcblocks, n)).max() < 1e-12


@pytest.mark.parametrize("Q,storage,tol_u,tol_rho", [(9, _lib.STORE_FP16, 1e-3, 1e-5), (9, _lib.STORE_BF16, 1e-2, 1e-4),
                                                     (19, _lib.STORE_FP16, 1e-3, 1e-5),
                                                     (27, _lib.STORE_BF16, 1e-2, 1e-4)])
def test_half_storage_vs_fp64_oracle(Q, storage, tol_u, tol_rho):
    N = 64 if Q == 9 else 16
    p = ldc_params(Q, N, storage=storage)
    F, Fo, _, _ = run_pair(p, 300 if Q == 9 else 100, fp64_oracle=True)
    dim = 2 if Q == 9 else 3
    n = (N // 4) ** dim
    pb, c, _ = lattice(Q)
    rho, u = macros_from_F(active(F, Q, p.n_maxcblocks, n), dim, Q, pb, c)
    rho_o, u_o = macros_from_F(active(Fo, Q, p.n_maxcblocks, n), dim, Q, pb, c)
    assert rel_l2(rho, rho_o) < tol_rho
    assert rel_l2(np.stack(u), np.stack(u_o)) < tol_u


@pytest.mark.parametrize("per", [(1, 0, 0), (0, 1, 0), (1, 1, 0)])
def test_periodic_2d(per):
    p = ldc_params(9, 32, extra=dict(PERIODIC_X=per[0], PERIODIC_Y=per[1], L_fy=0.5))
    p.n_maxcblocks = 8 * 4 + 3
    F, Fo, ints, oints = run_pair(p, 150)
    for k in ints:
        assert (ints[k] == oints[k]).all()
    assert np.abs(active(F, 9, p.n_maxcblocks, 32) - active(Fo, 9, p.n_maxcblocks, 32)).max() < 1e-5


def test_periodic_3d_fpsc_preset():
    p = ag.default_params(velocity_set=_lib.D3Q27, Nx=16, L_fy=0.5, L_fz=0.5, MAX_LEVELS_WALL=1,
                          MAX_LEVELS_INTERIOR=1, v0=1e-4, bc_preset=_lib.BC_FPSC3D, ic_preset=_lib.IC_UNIFORM,
                          ic_noise=0.01, seed=11, PERIODIC_Z=1, n_maxcblocks=20)
    F, Fo, _, _ = run_pair(p, 60)
    assert np.abs(active(F, 27, 20, 16) - active(Fo, 27, 20, 16)).max() < 2e-5


def test_root_grid_matches_brute_force():
    p = ag.default_params(velocity_set=_lib.D3Q19, Nx=16, L_fy=0.5, L_fz=0.75, MAX_LEVELS_WALL=1,
                          MAX_LEVELS_INTERIOR=1, PERIODIC_Y=1, n_maxcblocks=40)
    nb_exp, onb_exp = brute_root_grid(3, 16, 8, 12, (0, 1, 0))
    n = nb_exp.shape[1]
    with ag.Case(p) as c:
        nbr = c.dump(_lib.ARR_CBLOCK_ID_NBR).reshape(27, 40)
        onb = c.dump(_lib.ARR_CBLOCK_ID_ONB)
    assert (nbr[:, :n] == nb_exp).all() and (onb[:n] == onb_exp).all()


def test_graph_replay_bit_identical():
    p = ldc_params(9, 64)
    with ag.Case(p) as a, ag.Case(p) as b:
        a.set_ic(0)
        b.set_ic(0)
        for _ in range(40):
            a.advance()
        b.advance_n(20, use_graph=True)
        b.advance_n(20, use_graph=True)   # replay of the same graph
        a.sync()
        b.sync()
        assert np.array_equal(a.dump(_lib.ARR_F), b.dump(_lib.ARR_F))


@pytest.mark.parametrize("Q,storage", [(9, _lib.STORE_FP32), (19, _lib.STORE_FP16), (27, _lib.STORE_FP32),
                                       (9, _lib.STORE_FP64)])
def test_step_variants_bit_identical_and_autotune_pure(Q, storage):
    """The six step kernels (1 and 2 cells per thread, TMA-staged
    pipeline, one row of four cells per thread, root-level tiles, root-level
    push tiles) do the same
    arithmetic per cell, so their results agree bit for bit; autotuning leaves
    the state untouched."""
    N = 32 if Q == 9 else 12
    p = ldc_params(Q, N, storage=storage)
    out = []
    for v in (1, 2, 3, 4, 5, 6):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.set_tuning(v)
            c.advance_n(17, use_graph=False)
            c.sync()
            out.append(c.dump(_lib.ARR_F))
    for o in out[1:]:
        assert np.array_equal(out[0], o)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(5, use_graph=False)
        before = c.dump(_lib.ARR_F)
        r = c.autotune(0, reps=3)
        assert r["variant"] in (1, 2, 3, 4, 5, 6) and min(r["ms"]) > 0
        c.sync()
        assert np.array_equal(c.dump(_lib.ARR_F), before)   # tuning does not advance the state


@pytest.mark.parametrize("Q", [9, 19, 27])
def test_tma_pipeline_matches_oracle_many_chunks(Q):
    """The TMA pipeline at a size where every CTA cycles through its stage
    ring several times (chunk counts far above the persistent grid)."""
    N = 256 if Q == 9 else 48
    p = ldc_params(Q, N)
    F, Fo, _, _ = run_pair_variant(p, 20, 3)
    dim = 2 if Q == 9 else 3
    n = (N // 4) ** dim
    assert np.abs(active(F, Q, p.n_maxcblocks, n) - active(Fo, Q, p.n_maxcblocks, n)).max() < 1e-5


def run_pair_variant(p, steps, variant):
    from oracle.orc import OracleCase
    o = OracleCase(p, p.n_maxcblocks)
    o.set_ic(0)
    o.advance_n(steps)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.set_tuning(variant)
        c.advance_n(steps, use_graph=True)
        c.sync()
        F = c.dump(_lib.ARR_F)
    return F, o.dump(_lib.ARR_F), None, None


def test_deterministic():
    p = ldc_params(19, 16)
    out = []
    for _ in range(2):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.advance_n(30, use_graph=False)
            out.append(c.dump(_lib.ARR_F))
    assert np.array_equal(out[0], out[1])


def test_mass_momentum_fp64_matches_oracle():
    from oracle.orc import OracleCase
    p = ldc_params(9, 64, storage=_lib.STORE_FP64, extra=dict(PERIODIC_X=1, PERIODIC_Y=1, bc_preset=_lib.BC_NONE,
                                                              ic_preset=_lib.IC_UNIFORM, ic_noise=0.3, seed=3))
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    o.set_ic(0)
    with ag.Case(p) as c:
        c.set_ic(0)
        m0 = c.mass_momentum()
        assert np.allclose(m0, o.mass_momentum(), rtol=1e-13, atol=1e-12)
        c.advance_n(100, use_graph=False)
        m1 = c.mass_momentum()
    # periodic box, no walls: mass and momentum conserved to rounding
    assert abs(m1[0] - m0[0]) < 1e-10 * m0[0]
    assert np.abs(m1[1:] - m0[1:]).max() < 1e-9


def test_refresh_macros():
    p = ldc_params(27, 8)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(10, use_graph=False)
        c.refresh(0)
        M = c.dump(_lib.ARR_MACROS).reshape(4, -1)[:, : 8 * 64]
        F = c.dump(_lib.ARR_F).reshape(27, -1)[:, : 8 * 64]
    pb, cv, _ = lattice(27)
    rho, u = macros_from_F(F, 3, 27, pb, cv)
    assert np.abs(M[0] - rho).max() < 1e-6
    assert np.abs(M[1:] - np.stack(u)).max() < 1e-6


UNIFORM_CASES = [n for n in GOLDEN_CASES if not n.startswith(("amr_", "regrid_", "geom_", "restart_", "faces_", "les_"))]


@pytest.mark.skipif(not UNIFORM_CASES, reason="no reference dumps committed")
@pytest.mark.parametrize("name", UNIFORM_CASES)
def test_cuda_vs_reference_build(name):
    g = load_golden(name)
    p, steps = params_for_golden(g)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(steps, use_graph=False)
        c.sync()
        compare_to_golden(g, c.dump, 1e-5)


def test_large_grid_properties():
    """At benchmark scale (D2Q9 2048^2), where the oracle is too slow to run
    alongside: a closed cavity with plain bounce-back walls conserves its FP64
    mass to round-off and keeps zero momentum."""
    N = 2048
    p = ag.default_params(velocity_set=_lib.D2Q9, Nx=N, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=5e-4,
                          bc_preset=_lib.BC_NONE, n_maxcblocks=(N // 4) ** 2)
    with ag.Case(p) as c:
        c.set_ic(0)
        m0 = c.mass_momentum()
        c.advance_n(50, use_graph=True)
        m1 = c.mass_momentum()
    assert abs(m1[0] - m0[0]) < 1e-6 * m0[0]
    assert np.abs(m1[1:]).max() < 1e-6 * m0[0]


@pytest.mark.parametrize("storage,extra", [
    (_lib.STORE_FP16, dict(PERIODIC_X=1, PERIODIC_Y=1, bc_preset=_lib.BC_NONE, ic_preset=_lib.IC_UNIFORM,
                           ic_noise=0.3, seed=11)),
    (_lib.STORE_FP32, dict(PERIODIC_X=1, bc_preset=_lib.BC_NONE, ic_preset=_lib.IC_UNIFORM, ic_noise=0.2,
                           seed=5)),
    (_lib.STORE_BF16, dict()),
    (_lib.STORE_FP32, dict(Ny_factor=2)),
])
def test_tile_step_bit_identical(storage, extra):
    """The root-level tile steps (variant 5 and the push tiles of variant 6):
    fully periodic tiles (the select-free gather; every tile edge pushes into
    a neighbouring tile), a periodic channel with closed y walls, and
    lid-driven cavities (closed links, the lid hook) give the populations of
    one cell per thread bit for bit, with graph replay."""
    extra = dict(extra)
    ny = extra.pop("Ny_factor", 1)
    p = ldc_params(9, 64, storage=storage, extra=extra)
    if ny != 1:
        p.L_fy = float(ny)
        p.n_maxcblocks = 16 * 16 * ny
    out = []
    for v in (1, 5, 6):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.set_tuning(v)
            c.advance_n(40, use_graph=True)
            c.sync()
            out.append(c.dump(_lib.ARR_F))
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], out[2])


def test_tile_step_refused_swaps_bit_identical():
    """A lid-driven cavity driven hard enough (tau near 1/2, lid 0.3) that
    populations go non-positive at the lid corners: the reference's stream
    guard refuses those swaps.  The tile step decides them locally, the push
    tiles record them (in and across tiles) in the fix-up list, and both must
    match the push variants bit for bit."""
    p = ldc_params(9, 64, extra=dict(v0=1e-7, u_ref=0.3))
    out, neg = [], 0
    for v in (1, 5, 6):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.set_tuning(v)
            for _ in range(6):
                c.advance_n(5, use_graph=False)
                F = c.dump(_lib.ARR_F)
                neg += int((F.reshape(9, -1) <= 0).sum())
            out.append(F)
    assert neg > 0, "the case did not produce a non-positive population"
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], out[2])


def test_mass_momentum_async_equals_sync():
    """The enqueued FP64 sums land in host memory after sync and equal the
    blocking call's (same kernels, fixed reduction order)."""
    p = ldc_params(19, 16, storage=_lib.STORE_FP16)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(12, use_graph=True)
        out = np.full(4, np.nan)
        c.mass_momentum_async(out)
        c.sync()
        ref = c.mass_momentum()
        assert np.array_equal(out[:4], ref)
        assert abs(out[0] - 16 ** 3) < 1e-6 * 16 ** 3


@pytest.mark.parametrize("storage", [_lib.STORE_FP16, _lib.STORE_FP32])
def test_dump_load_round_trip_many_chunks(storage):
    """Device-side layout conversion through the staging buffer over several
    chunks (65,536 blocks): dump -> load into a fresh case -> dump is the
    identity, and both cases then step bit for bit alike (round-to-nearest:
    stochastic rounding also depends on each case's own step counter)."""
    p = ldc_params(9, 1024, storage=storage, extra=dict(half_rounding=_lib.ROUND_NEAREST))
    with ag.Case(p) as a, ag.Case(p) as b:
        a.set_ic(0)
        a.advance_n(5, use_graph=True)
        Fa = a.dump(_lib.ARR_F)
        b.load(_lib.ARR_F, Fa)
        assert np.array_equal(b.dump(_lib.ARR_F), Fa)
        a.advance_n(3, use_graph=True)
        b.advance_n(3, use_graph=True)
        assert np.array_equal(a.dump(_lib.ARR_F), b.dump(_lib.ARR_F))
