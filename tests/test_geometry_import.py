"""Geometry import on the host (agal_geometry_read_stl / _read_text /
_refine_length, the reference's G_ImportSTL_ASCII, geometry.txt primitives and
G_RefineFaces_Length) against the face lists the reference's own build holds
after its import (tests/golden/geom_*.npz and faces_*.npz)."""
import json

import numpy as np
import pytest

from test_oracle import GOLDEN
from test_oracle_geometry import GEOM_CASES

import agal_b200 as ag
from agal_b200.geometry import icosphere, import_stl, import_text, refine_length, write_stl_ascii


def params_of(keys: dict):
    return ag.default_params(**{k: v for k, v in keys.items() if k not in ("G_FILENAME",)})


@pytest.mark.parametrize("name", GEOM_CASES)
def test_stl_import_and_length_refinement_match_the_reference(tmp_path, name):
    g = np.load(GOLDEN / f"{name}.npz")
    sphere = json.loads(str(g["sphere"]))
    stl = tmp_path / "sphere.stl"
    write_stl_ascii(stl, icosphere(sphere[0], sphere[1], tuple(sphere[2]), seed=sphere[3]))
    faces = refine_length(params_of(json.loads(str(g["case_keys"]))), import_stl(stl))
    assert np.array_equal(faces, g["faces_soa"].T)


def _faces_fixture(name):
    path = GOLDEN / f"{name}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated")
    return np.load(path)


def test_split_faces_match_the_reference(tmp_path):
    """A coarse icosphere whose faces are longer than the finest bin spacing:
    split at the midpoints, pieces in the reference's order."""
    g = _faces_fixture("faces_stl_split")
    sphere = json.loads(str(g["sphere"]))
    stl = tmp_path / "sphere.stl"
    raw = icosphere(sphere[0], sphere[1], tuple(sphere[2]), seed=sphere[3])
    write_stl_ascii(stl, raw)
    faces = refine_length(params_of(json.loads(str(g["case_keys"]))), import_stl(stl))
    assert len(faces) > len(raw)
    assert np.array_equal(faces, g["faces_soa"].T)


def test_text_primitives_match_the_reference(tmp_path):
    """PRISM (corner and centre forms) and a latitude-longitude SPHERE from a
    geometry.txt, after the length refinement."""
    g = _faces_fixture("faces_text_primitives")
    txt = tmp_path / "geometry.txt"
    txt.write_text(str(g["geometry_txt"]))
    p = params_of(json.loads(str(g["case_keys"])))
    faces = refine_length(p, import_text(p, txt))
    ref = g["faces_soa"].T
    assert faces.shape == ref.shape
    assert np.array_equal(faces, ref)


def test_stl_reader_drops_degenerate_facets(tmp_path):
    f = icosphere(1, 0.2, (0.5, 0.5, 0.5), seed=1).reshape(-1, 9)
    bad = f.copy()
    bad[3, 3:6] = bad[3, 0:3]            # vertex 2 == vertex 1
    stl = tmp_path / "d.stl"
    write_stl_ascii(stl, bad.reshape(-1, 3, 3))
    got = import_stl(stl)
    assert len(got) == len(f) - 1
    assert np.array_equal(got, np.delete(bad, 3, axis=0))


def test_text_2d_shapes_are_refused(tmp_path):
    txt = tmp_path / "geometry.txt"
    txt.write_text("CIRCLE 32 0.5 0.5 0.1\nEND\n")
    with pytest.raises(ag.AgalError):
        import_text(ag.default_params(), txt)
