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

LES_CASES = {"les_d3q19_ldc16_smag": 1, "les_d3q19_ldc16_wale": 2, "les_d3q19_ldc16_vreman": 3}
TOL_U = 1e-4          # relative L2 of the velocity after 200 steps


def run(g, model):
    p, steps = params_for_golden(g)
    p.S_LES = model
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


@pytest.mark.gpu
@pytest.mark.parametrize("name,model", sorted(LES_CASES.items()))
def test_les_matches_the_reference_build(name, model):
    g = np.load(GOLDEN / f"{name}.npz")
    Q = int(g["Q"])
    Fr = np.transpose(g["F"][:, :Q, :], (1, 0, 2)).reshape(Q, -1)
    rho_r, u_r = macros(g, Fr)
    rho, u = macros(g, run(g, model))
    _, u0 = macros(g, run(g, 0))
    e, e0 = rel_l2(u, u_r), rel_l2(u0, u_r)
    assert rel_l2(rho, rho_r) < TOL_U
    assert e < TOL_U, (e, e0)
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
