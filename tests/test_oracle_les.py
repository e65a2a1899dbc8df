"""The LES eddy-viscosity restatement (oracle/les.py) against the reference's
own build: its LES fixtures hold, after the last step, the velocity rows
written by Cu_CollideLES and the eddy viscosity that Cu_ComputeEddyViscosity
computed from the same state (row Q + 4 of the field)."""
import json

import numpy as np
import pytest

from test_oracle import GOLDEN

from oracle.les import eddy_viscosity

LES_CASES = {"les_d3q19_ldc16_smag": 1, "les_d3q19_ldc16_wale": 2, "les_d3q19_ldc16_vreman": 3,
             "les_d2q9_ldc64_smag": 1, "les_d2q9_ldc64_wale": 2, "les_d2q9_ldc64_vreman": 3}


@pytest.mark.parametrize("name,model", sorted(LES_CASES.items()))
def test_eddy_viscosity_restatement_matches_the_reference(name, model):
    g = np.load(GOLDEN / f"{name}.npz")
    dim, Q = int(g["dim"]), int(g["Q"])
    F = g["F"].astype(np.float64)
    assert F.shape[1] == Q + 5                # the harness sizes LES fields to row Q + 4
    dx = 1.0 / json.loads(str(g["case_keys"]))["Nx"]
    nu = eddy_viscosity(F[:, Q + 1:Q + 1 + dim, :], dx, model, dim)
    ref = F[:, Q + 4, :]
    v0 = json.loads(str(g["case_keys"]))["v0"]
    assert ref.max() > 0.1 * v0               # the model is active in this flow
    assert np.abs(nu - ref).max() < 2e-4 * ref.max(), np.abs(nu - ref).max() / ref.max()
