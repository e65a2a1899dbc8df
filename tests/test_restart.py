"""Checkpoint / restart in the reference's restart.bin format
(Mesh::M_Restart, mesh_restart.cu:45-225).

The fixture tests/golden/restart_d2q9_wall2_sol3.npz holds the reference's own
restart.bin of a two-level-wall, three-level-solution D2Q9 cavity after 200
steps (written by the reference build through its M_Restart SAVE) and the
harness dump of the same state.  On the CPU the documented layout is parsed
from the reference's bytes and checked against that dump; on the GPU the
library loads the reference's file, writes it back byte for byte, and a run
interrupted by save / load continues bit for bit as the uninterrupted run.
"""
import numpy as np
import pytest

from test_oracle import GOLDEN, params_for_golden

FIXTURE = GOLDEN / "restart_d2q9_wall2_sol3.npz"
pytestmark_fixture = pytest.mark.skipif(not FIXTURE.exists(), reason="restart fixture not generated")


def parse_restart(buf: bytes, dim: int, Q: int, Qmax: int, MC: int, ML: int, real=np.float32) -> dict:
    """The documented restart.bin layout, read with numpy."""
    pos = 0

    def take(dt, n):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=n, offset=pos)
        pos += a.nbytes
        return a

    r = {"n_maxcblocks": int(take(np.int32, 1)[0]), "n_ids": take(np.int32, ML + 1).copy(),
         "n_gaps": int(take(np.int32, 1)[0]), "id_max": take(np.int32, ML + 1).copy()}
    cb = int(take(np.int32, 1)[0])
    cells = int(take(np.int64, 1)[0])
    r.update(cblocks_id_max=cb, cells_id_max=cells, n_ids_probed=int(take(np.int32, 1)[0]),
             iter=int(take(np.int32, 1)[0]))
    r["id_set"] = [take(np.int32, int(r["n_ids"][L])) for L in range(ML)]
    r["gap_set"] = take(np.int32, r["n_gaps"])
    r["cmask"] = take(np.int32, cells)
    r["fX"] = np.stack([take(real, cb) for _ in range(dim)], axis=1)
    r["bmask"] = take(np.int32, cb)
    nbr, child = [], []
    for _ in range(Qmax):
        nbr.append(take(np.int32, cb))
        child.append(take(np.int32, cb))
    r["nbr"], r["nbr_child"] = np.stack(nbr, axis=1), np.stack(child, axis=1)
    r["onb"], r["ref"], r["level"] = take(np.int32, cb), take(np.int32, cb), take(np.int32, cb)
    r["F_offset"] = pos
    r["F"] = np.stack([take(real, cells) for _ in range(Q)])
    r["macros_offset"] = pos
    r["macros"] = np.stack([take(real, cells) for _ in range(dim + 1)])
    r["probed_offset"] = pos
    r["probed"] = take(real, dim * r["n_ids_probed"] * MC)
    r["mean_offset"] = pos
    r["mean"] = take(real, (dim + 1) * int(r["n_ids"][0]) * MC)
    r["end"] = pos
    return r


def fixture():
    """The fixture with the reference's restart.bin rebuilt byte for byte
    (its gap stack is stored as first value + differences)."""
    import hashlib
    d = np.load(FIXTURE, allow_pickle=False)
    g = {k: d[k] for k in d.files}
    n = int(g["restart_n_gaps"])
    gaps = (np.concatenate([[int(g["restart_gap_first"])], g["restart_gap_diff"]]).cumsum()[:n]
            if n else np.zeros(0)).astype(np.int32)
    b = g["restart_head"].tobytes() + gaps.tobytes() + g["restart_tail"].tobytes()
    assert hashlib.sha256(b).hexdigest() == str(g["restart_sha256"])
    g["restart_bin"] = np.frombuffer(b, dtype=np.uint8)
    return g


@pytestmark_fixture
def test_reference_restart_layout_matches_its_dump():
    g = fixture()
    buf = g["restart_bin"].tobytes()
    dim, Q, Qmax, MC, ML = (int(g[k]) for k in ("dim", "Q", "Qmax", "MC", "max_levels"))
    r = parse_restart(buf, dim, Q, Qmax, MC, ML)
    assert r["end"] == len(buf)
    assert r["n_maxcblocks"] == int(g["n_maxcblocks"])
    assert np.array_equal(r["n_ids"], g["n_ids"]) and np.array_equal(r["id_max"], g["id_max"])
    assert r["n_gaps"] == int(g["n_gaps"]) and r["iter"] == int(g["steps"]) - 1
    assert r["n_ids_probed"] == 16          # every 4th root block per axis of the 16 x 16 root grid
    assert r["cblocks_id_max"] == int(g["id_max"][ML]) and r["cells_id_max"] == r["cblocks_id_max"] * MC
    for L in range(ML):
        assert np.array_equal(r["id_set"][L], g[f"id_set_{L}"])
    tail = g["gaps_tail"]
    assert np.array_equal(r["gap_set"][r["n_gaps"] - len(tail):], tail)
    b = g["blocks"].astype(np.int64)
    assert np.array_equal(r["cmask"].reshape(-1, MC)[b], g["cmask"])
    assert np.array_equal(r["fX"][b], g["fX"])
    for k in ("bmask", "onb", "ref", "level"):
        assert np.array_equal(r[k][b], g[k][:, 0]), k
    assert np.array_equal(r["nbr"][b], g["nbr"]) and np.array_equal(r["nbr_child"][b], g["nbr_child"])
    F = r["F"].reshape(Q, -1, MC)[:, b, :].transpose(1, 0, 2)
    assert np.array_equal(F, g["F"][:, :Q, :])


@pytestmark_fixture
@pytest.mark.gpu
def test_library_reads_and_writes_the_reference_file(tmp_path):
    import agal_b200 as ag
    from agal_b200 import _lib
    g = fixture()
    p, _ = params_for_golden(g)
    p.n_maxcblocks = int(g["n_maxcblocks"])
    src = tmp_path / "restart.bin"
    src.write_bytes(g["restart_bin"].tobytes())
    with ag.Case(p) as c:
        assert c.restart_load(src) == int(g["steps"]) - 1
        cnt = c.counts()
        assert cnt["n_ids"] == [int(x) for x in g["n_ids"]] and cnt["n_gaps"] == int(g["n_gaps"])
        MC, Q, nmb = int(g["MC"]), int(g["Q"]), p.n_maxcblocks
        b = g["blocks"].astype(np.int64)
        assert np.array_equal(c.dump(_lib.ARR_CELLS_ID_MASK).reshape(nmb, MC)[b], g["cmask"])
        assert np.array_equal(c.dump(_lib.ARR_CBLOCK_ID_NBR).reshape(-1, nmb)[:, b].T, g["nbr"])
        F = c.dump(_lib.ARR_F).reshape(Q, nmb, MC)[:, b, :].transpose(1, 0, 2)
        assert np.array_equal(F.astype(np.float32), g["F"][:, :Q, :])
        out = tmp_path / "again.bin"
        c.restart_save(out, int(g["steps"]) - 1)
        a, ref = out.read_bytes(), g["restart_bin"].tobytes()
        dim, Qmax, ML = int(g["dim"]), int(g["Qmax"]), int(g["max_levels"])
        r = parse_restart(ref, dim, Q, Qmax, MC, ML)
        # Identical but for the macro rows (the reference's hold its last
        # collide's macros, this library's those of the saved populations) and
        # the probe velocities and running mean (uninitialised host arrays in
        # the reference, zeros here).
        assert len(a) == len(ref)
        assert a[: r["macros_offset"]] == ref[: r["macros_offset"]]
        ra = parse_restart(a, dim, Q, Qmax, MC, ML)
        assert ra["n_ids_probed"] == r["n_ids_probed"]
        # this library's macro rows are rho and u of the populations it wrote
        from helpers import lattice
        pb, cv, _ = lattice(Q)
        F64 = ra["F"].astype(np.float64)
        rho = F64.sum(axis=0)
        assert np.allclose(ra["macros"][0], rho, rtol=1e-6)
        for d in range(dim):
            ud = (np.asarray(cv[d][:Q])[np.asarray(pb)[:Q]][:, None] * F64).sum(axis=0) / rho
            assert np.allclose(ra["macros"][1 + d], ud, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["STORE_FP32", "STORE_FP16", "STORE_FP64"])
def test_save_load_continues_bit_for_bit(tmp_path, storage):
    """40 steps, save, a fresh case loads and runs 24 more: every mesh array
    and the populations equal those of 64 uninterrupted steps (the regrids
    every 8 steps included: the coarse-step counter, which also seeds the
    stochastic rounding of FP16, is restored).  FP16 populations agree to the
    FP32 rounding of the file's f = w + g."""
    import agal_b200 as ag
    from agal_b200 import _lib
    from test_gpu_amr import amr_params
    p = amr_params(9, 32, storage=getattr(_lib, storage), S_CRITERION=_lib.CRITERION_PERCENTILE, P_REFINE=8,
                   MAX_LEVELS_INTERIOR=3, v0=5e-4)
    arrays = (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR, _lib.ARR_CBLOCK_ID_NBR_CHILD,
              _lib.ARR_CBLOCK_ID_REF, _lib.ARR_CBLOCK_LEVEL, _lib.ARR_ID_SET, _lib.ARR_GAP_SET, _lib.ARR_F)
    with ag.Case(p) as a, ag.Case(p) as b:
        for c in (a, b):
            c.set_ic(0)
            c.refine_near_wall()
        a.advance_n(64)
        b.advance_n(40)
        b.restart_save(tmp_path / "r.bin", 39)
        with ag.Case(p) as c:
            assert c.restart_load(tmp_path / "r.bin") == 39
            c.advance_n(24)
            a.sync()
            c.sync()
            assert c.counts()["n_ids"] == a.counts()["n_ids"] and c.counts()["n_gaps"] == a.counts()["n_gaps"]
            assert c.refine_stats()["iter"] == a.refine_stats()["iter"]
            for k in arrays:
                if k == _lib.ARR_F and storage == "STORE_FP16":
                    # the file holds f = w + g in FP32, which near the weights
                    # keeps fewer bits than the scaled FP16 offset g
                    d = np.abs(c.dump(k) - a.dump(k))
                    assert d.max() < 1e-4 and np.sqrt((d ** 2).mean()) < 1e-6, (d.max(), np.sqrt((d ** 2).mean()))
                else:
                    assert np.array_equal(c.dump(k), a.dump(k)), k
