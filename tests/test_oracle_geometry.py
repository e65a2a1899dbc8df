"""The CPU oracle's geometry chain against the reference build's own dumps.

Fixtures tests/golden/geom_*.npz were written by the reference (KhodrJ/AGAL)
compiled from its sources with oracle/ref_harness (REF_GEOM=1): a seeded
icosphere imported as ASCII STL (geometry_import.cu), binned
(geometry_bins_gpu.cu), voxelized with near-wall refinement
(mesh_voxelizer*.cu), link lengths (mesh_voxelizer_links.cu), then flow past
it with the interpolated bounce-back (solver_lbm_kernels.cu:693-887) and the
MEA forces (solver_lbm_kernels_forces.cu:324-599).

Integer results (bins, masks, block states, wall-block slots) and the FP32
link lengths are compared bit for bit; populations and force partials at the
FP32 round-off floor of these short runs.
"""
import json

import numpy as np
import pytest

import agal_b200 as ag
from agal_b200 import _lib
from agal_b200.geometry import face_soa, icosphere, read_stl_ascii, write_stl_ascii

from test_oracle import GOLDEN, params_for_golden

GEOM_CASES = ["geom_d3q19_uniform", "geom_d3q27_wall2_bb", "geom_d3q19_wall3_bouzidi"]


def geom_params(g):
    p, steps = params_for_golden(g)
    p.bc_preset = _lib.BC_FPSC3D
    p.ic_preset = _lib.IC_UNIFORM
    p.u_ref = 0.05
    return p, steps


def faces_of(g):
    return np.ascontiguousarray(g["faces_soa"].T)


@pytest.fixture(scope="module", params=GEOM_CASES)
def geom_run(request):
    """Oracle run of one fixture: bins, near-wall voxelization, the steps."""
    from oracle.orc import OracleCase
    g = dict(np.load(GOLDEN / f"{request.param}.npz"))
    p, steps = geom_params(g)
    o = OracleCase(p, p.n_maxcblocks)
    o.set_geometry(faces_of(g))
    bins = [o.bins(L) for L in range(int(g["n_bin_levels"]))]
    bins_md = o.bins(-1)
    o.set_ic(0)
    o.refine_near_wall()
    pre = {k: o.dump(a) for k, a in [("cmask", _lib.ARR_CELLS_ID_MASK), ("bmask", _lib.ARR_CBLOCK_ID_MASK),
                                     ("ref", _lib.ARR_CBLOCK_ID_REF), ("onb", _lib.ARR_CBLOCK_ID_ONB),
                                     ("nbr", _lib.ARR_CBLOCK_ID_NBR), ("onb_solid", _lib.ARR_CBLOCK_ID_ONB_SOLID),
                                     ("X_b", _lib.ARR_CELLS_F_X_B)]}
    counts = o.counts()
    gcounts = o.geometry_counts()
    o.advance_n(steps)
    post = {"Ff": o.dump(_lib.ARR_CBLOCK_F_FF), "F": o.dump(_lib.ARR_F)}
    yield dict(g=g, p=p, bins=bins, bins_md=bins_md, pre=pre, post=post, counts=counts, gcounts=gcounts)
    o.close()


def test_fixture_faces_are_the_seeded_icosphere():
    """The reference imported the generator's STL without splitting faces."""
    for name in GEOM_CASES:
        g = np.load(GOLDEN / f"{name}.npz")
        sub, r, centre, seed = json.loads(str(g["sphere"]))
        assert np.array_equal(face_soa(icosphere(sub, r, centre, seed)), g["faces_soa"])


def test_stl_round_trip_and_degenerate_faces(tmp_path):
    f = icosphere(2, 0.2, (0.5, 0.5, 0.5), seed=1)
    bad = f[:2].copy()
    bad[0, 1] = bad[0, 0]                      # two equal vertices: dropped on import
    path = tmp_path / "s.stl"
    write_stl_ascii(path, np.concatenate([f, bad]))
    back = read_stl_ascii(path)
    assert back.shape == (len(f) + 1, 3, 3)
    assert np.array_equal(back[: len(f)], f)


def test_bins_bit_exact(geom_run):
    g = geom_run["g"]
    for L, (dens, n, N, ids) in enumerate(geom_run["bins"]):
        assert dens == int(g[f"bins_density_{L}"])
        assert np.array_equal(n, g[f"bins_n_{L}"]), L
        assert np.array_equal(N, g[f"bins_N_{L}"]), L
        assert np.array_equal(ids, g[f"bins_ids_{L}"]), L
    dens, n, N, ids = geom_run["bins_md"]
    assert dens == int(g["bins_md_density"])
    assert np.array_equal(n, g["bins_md_n"]) and np.array_equal(N, g["bins_md_N"])
    assert np.array_equal(ids, g["bins_md_ids"])


def test_voxelization_bit_exact(geom_run):
    g, p, pre = geom_run["g"], geom_run["p"], geom_run["pre"]
    nmb, MC, Qmax = p.n_maxcblocks, int(g["MC"]), int(g["Qmax"])
    blocks = g["blocks"].astype(np.int64)
    ml = int(g["max_levels"])
    assert geom_run["counts"]["n_ids"][:ml] == [int(v) for v in g["n_ids"][:ml]]
    assert np.array_equal(pre["cmask"].reshape(nmb, MC)[blocks], g["cmask"])
    for key in ("bmask", "ref", "onb"):
        assert np.array_equal(pre[key][blocks], g[key][:, 0]), key
    assert np.array_equal(pre["nbr"].reshape(Qmax, nmb)[:, blocks].T, g["nbr"])
    assert np.array_equal(pre["onb_solid"][blocks], g["onb_solid"])
    gc = geom_run["gcounts"]
    assert (gc["n_solida"], gc["n_solidb"], gc["n_maxcells_b"]) == (int(g["n_solida"]), int(g["n_solidb"]),
                                                                     int(g["n_maxcells_b"]))
    # Every voxelizer cell state is present: solid, boundary and fluid.
    assert {-1, -6, 0} <= set(np.unique(g["cmask"]).tolist())


def test_link_lengths_bit_exact(geom_run):
    g, pre = geom_run["g"], geom_run["pre"]
    xb = pre["X_b"].reshape(int(g["Qmax"]), -1)
    assert xb.shape == g["cells_f_X_b"].shape
    assert np.array_equal(xb, g["cells_f_X_b"])
    assert (xb > 0).sum() > 100


def test_wall_flow_and_forces_at_fp32_floor(geom_run):
    g, p, post = geom_run["g"], geom_run["p"], geom_run["post"]
    nmb, MC, Q = p.n_maxcblocks, int(g["MC"]), int(g["Q"])
    blocks = g["blocks"].astype(np.int64)
    fb = blocks[g["F_blocks"]] if "F_blocks" in g else blocks
    F = post["F"].reshape(Q, nmb, MC)[:, fb, :].transpose(1, 0, 2)
    # FP32 round-off of 16-24 steps: the reference and the oracle round the
    # same formulas in a different order (fused multiply-adds there).
    assert np.abs(F - g["F"][:, :Q, :].astype(np.float64)).max() < 2e-6
    Ff = post["Ff"].reshape(6, nmb)[:, blocks].T
    ref = g["Ff"].astype(np.float64)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(Ff - ref).max() < 5e-6 * scale
    for d in range(3):
        s, r = Ff[:, 2 * d].sum(), ref[:, 2 * d].sum()
        assert abs(s - r) < 1e-5 * np.abs(ref[:, 2 * d]).sum() + 1e-12
