"""D3Q19 multiple-relaxation-time collision (no live kernel in the reference:
the moment basis and equilibria of its legacy MRT kernel, restated by the
oracle).  FP64 CUDA vs FP64 oracle within 1e-12; FP32 within 1e-5 relative L2
of rho/u of the FP64 oracle; FP16 weight-offset storage within 1e-3 (u)."""
import numpy as np
import pytest

from helpers import lattice, macros_from_F, rel_l2

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu


def mrt_params(N=16, storage=_lib.STORE_FP64, **kw):
    base = dict(velocity_set=_lib.D3Q19, Nx=N, MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=1.25e-4,
                bc_preset=_lib.BC_LDC3D, collision=_lib.MRT, s1=1.2, s2=1.2, s3=1.2, s5=1.2, s6=1.2,
                storage=storage, n_maxcblocks=(N // 4) ** 3 + 5)
    base.update(kw)
    return ag.default_params(**base)


def run(p, steps, fp64_oracle):
    from oracle.orc import OracleCase
    o = OracleCase(p, p.n_maxcblocks, fp64=fp64_oracle)
    o.set_ic(0)
    o.advance_n(steps)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(steps, use_graph=True)
        c.sync()
        F = c.dump(_lib.ARR_F)
    return F, o.dump(_lib.ARR_F)


def test_mrt_fp64_matches_oracle():
    p = mrt_params(12)
    F, Fo = run(p, 100, True)
    n = 27 * 64
    assert np.abs(F.reshape(19, -1)[:, :n] - Fo.reshape(19, -1)[:, :n]).max() < 1e-12


def test_mrt_fp32_within_its_round_off_floor():
    """FP32 CUDA no further from the FP64 oracle than twice the FP32 oracle's
    own distance (FP32 round-off after 200 steps is ~1e-5 in u)."""
    from oracle.orc import OracleCase
    p = mrt_params(16, storage=_lib.STORE_FP32)
    F, Fo64 = run(p, 200, True)
    o32 = OracleCase(p, p.n_maxcblocks)
    o32.set_ic(0)
    o32.advance_n(200)
    n = 64 * 64
    pb, cv, _ = lattice(19)
    _, u = macros_from_F(F.reshape(19, -1)[:, :n], 3, 19, pb, cv)
    _, u64 = macros_from_F(Fo64.reshape(19, -1)[:, :n], 3, 19, pb, cv)
    _, u32 = macros_from_F(o32.dump(_lib.ARR_F).reshape(19, -1)[:, :n], 3, 19, pb, cv)
    e_cuda, e_orc = rel_l2(np.stack(u), np.stack(u64)), rel_l2(np.stack(u32), np.stack(u64))
    assert e_cuda <= 2 * e_orc + 1e-7, (e_cuda, e_orc)


@pytest.mark.parametrize("storage,tol_u", [(_lib.STORE_FP16, 1e-3), (_lib.STORE_BF16, 1e-2)])
def test_mrt_half_storage_vs_fp64_oracle(storage, tol_u):
    p = mrt_params(16, storage=storage)
    F, Fo = run(p, 200, True)
    n = 64 * 64
    pb, cv, _ = lattice(19)
    rho, u = macros_from_F(F.reshape(19, -1)[:, :n], 3, 19, pb, cv)
    ro, uo = macros_from_F(Fo.reshape(19, -1)[:, :n], 3, 19, pb, cv)
    assert rel_l2(np.stack(u), np.stack(uo)) < tol_u
    assert rel_l2(rho, ro) < tol_u * 1e-2


@pytest.mark.parametrize("storage", [_lib.STORE_FP32, _lib.STORE_FP16])
def test_mrt_step_variants_bit_identical(storage):
    p = mrt_params(12, storage=storage)
    out = []
    for v in (1, 2, 3, 4, 5, 6):
        with ag.Case(p) as c:
            c.set_ic(0)
            c.set_tuning(v)
            c.advance_n(23, use_graph=False)
            c.sync()
            out.append(c.dump(_lib.ARR_F))
    assert all(np.array_equal(out[0], o) for o in out[1:])


def test_mrt_two_levels_fp64_matches_oracle():
    """MRT in the multi-level recursion (box region, 2 levels)."""
    from oracle.orc import OracleCase
    p = mrt_params(16, MAX_LEVELS_WALL=2, region_preset=_lib.REGION_BOX, n_maxcblocks=64 + 512 + 64)
    o = OracleCase(p, p.n_maxcblocks, fp64=True)
    o.set_ic(0)
    o.refine_near_wall()
    o.advance_n(30)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(30, use_graph=True)
        c.sync()
        assert c.counts()["n_ids"] == o.counts()["n_ids"]
        ids = c.dump(_lib.ARR_ID_SET).reshape(-1, p.n_maxcblocks)
        cnt = c.counts()["n_ids"]
        blocks = np.concatenate([ids[L, : cnt[L]] for L in range(2)])
        F = c.dump(_lib.ARR_F).reshape(19, p.n_maxcblocks, 64)[:, blocks]
    Fo = o.dump(_lib.ARR_F).reshape(19, p.n_maxcblocks, 64)[:, blocks]
    assert np.abs(F - Fo).max() < 1e-12
