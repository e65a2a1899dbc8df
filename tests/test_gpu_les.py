"""LES (S_LES = 1 Smagorinsky, 2 WALE, 3 Vreman) on the GPU against the
reference's own LES builds: a 16^3 D3Q19 lid-driven cavity, one level, 200
steps from rest (Cu_ComputeEddyViscosity + Cu_CollideLES,
solver_lbm_kernels_les.cu:460-600, solver_lbm_kernels.cu:293-380).

The velocity field after 200 steps must agree with the reference's within
the FP32 floor of two implementations that round differently, and lie far
closer to it than the same run without the model does."""
import numpy as np
import pytest

from helpers import lattice, macros_from_F, rel_l2
from test_oracle import GOLDEN, params_for_golden

import agal_b200 as ag
from agal_b200 import _lib

LES_CASES = {"les_d3q19_ldc16_smag": 1, "les_d3q19_ldc16_wale": 2, "les_d3q19_ldc16_vreman": 3,
             "les_d2q9_ldc64_smag": 1, "les_d2q9_ldc64_wale": 2, "les_d2q9_ldc64_vreman": 3}
TOL_U = 1e-4          # relative L2 of the velocity after 200 (3D) / 400 (2D) steps
TOL_U_HALF = 2e-3     # the same with FP16 weight offsets (stochastic rounding)


def run(g, model, storage=None):
    p, steps = params_for_golden(g)
    p.S_LES = model
    if storage is not None:
        p.storage = storage
    Q, MC = int(g["Q"]), int(g["MC"])
    with ag.Case(p) as c:
        c.set_ic(0)
        c.advance_n(steps, use_graph=False)
        c.sync()
        F = c.dump(_lib.ARR_F)
        nmb = len(c.dump(_lib.ARR_CBLOCK_ID_ONB))
    blocks = g["blocks"].astype(np.int64)
    return F.reshape(Q, nmb, MC)[:, blocks, :].reshape(Q, -1)


def macros(g, F):
    dim, Q = int(g["dim"]), int(g["Q"])
    pb, c, _ = lattice(Q)
    rho, u = macros_from_F(F.astype(np.float64), dim, Q, pb, c)
    return rho, np.stack(u)


def fixture(name):
    path = GOLDEN / f"{name}.npz"
    if not path.exists():
        pytest.skip(f"{name} fixture not generated")
    return np.load(path)


@pytest.mark.gpu
@pytest.mark.parametrize("name,model", sorted(LES_CASES.items()))
def test_les_matches_the_reference_build(name, model):
    """FP32 velocity within max(TOL_U, 3 x this library's own FP32-vs-FP64
    distance) of the reference build's: two FP32 implementations that round
    differently drift apart by about their own round-off, which grows with
    the Reynolds number and the step count (2D: Re 2000, 400 steps)."""
    g = fixture(name)
    Q = int(g["Q"])
    Fr = np.transpose(g["F"][:, :Q, :], (1, 0, 2)).reshape(Q, -1)
    rho_r, u_r = macros(g, Fr)
    rho, u = macros(g, run(g, model))
    _, u64 = macros(g, run(g, model, _lib.STORE_FP64))
    _, u0 = macros(g, run(g, 0))
    e, e0, floor = rel_l2(u, u_r), rel_l2(u0, u_r), rel_l2(u, u64)
    print(f"{name}: u rel L2 vs reference {e:.3e}, FP32-vs-FP64 floor {floor:.3e}, no model {e0:.3e}")
    tol = max(TOL_U, 3 * floor)
    assert rel_l2(rho, rho_r) < tol
    assert e < tol, (e, floor, e0)
    assert e0 > 20 * e, (e, e0)      # the model changes the flow well beyond the agreement


@pytest.mark.gpu
def test_les_outside_its_scope_is_refused():
    g = np.load(GOLDEN / "les_d3q19_ldc16_smag.npz")
    p, _ = params_for_golden(g)
    p.S_LES = 1
    p.MAX_LEVELS_INTERIOR = 2
    with pytest.raises(ag.AgalError):
        ag.Case(p)
    p.MAX_LEVELS_INTERIOR = 1
    p.S_LES = 4
    with pytest.raises(ag.AgalError):
        ag.Case(p)


@pytest.mark.gpu
@pytest.mark.parametrize("name,model", [("les_d3q19_ldc16_smag", 1), ("les_d2q9_ldc64_wale", 2)])
@pytest.mark.parametrize("storage", ["STORE_FP16", "STORE_BF16"])
def test_les_half_storage_near_the_reference(name, model, storage):
    """FP16 / BF16 weight offsets: the eddy viscosity reads the decoded
    populations and the per-cell relaxation writes rounded offsets.  The
    velocity's distance from the reference build is the half-precision
    floor -- this library's own half-vs-FP64 distance on the same case -- and
    no more, and the model's effect stays well above it."""
    g = fixture(name)
    Q = int(g["Q"])
    Fr = np.transpose(g["F"][:, :Q, :], (1, 0, 2)).reshape(Q, -1)
    _, u_r = macros(g, Fr)
    st = getattr(_lib, storage)
    _, u = macros(g, run(g, model, st))
    _, u64 = macros(g, run(g, model, _lib.STORE_FP64))
    _, u0 = macros(g, run(g, 0, st))
    e, e0, floor = rel_l2(u, u_r), rel_l2(u0, u_r), rel_l2(u, u64)
    print(f"{name} {storage}: u rel L2 vs reference {e:.3e}, vs FP64 {floor:.3e}, no model {e0:.3e}")
    if name.startswith("les_d3q19"):
        assert e < (TOL_U_HALF if storage == "STORE_FP16" else 8 * TOL_U_HALF), (e, floor)
    assert e < 1.2 * floor + 2 * TOL_U, (e, floor)
    assert e0 > 3 * e, (e, e0)
