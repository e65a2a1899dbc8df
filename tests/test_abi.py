"""C-ABI surface: the library loads without a GPU, exports exactly the entry
points include/agal_b200.h declares, and the parameter layer follows the
reference's Parser (inc/parser.h:58-183)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(agal_[a-z0-9_]+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_exports_match_header(agal_lib):
    from agal_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln and ln.split()[-1].startswith("agal_")})
    declared = declared_functions()
    assert declared, "no declarations parsed"
    assert exported == declared


def test_every_declared_symbol_resolves(agal_lib):
    for name in declared_functions():
        assert getattr(agal_lib, name) is not None


def test_python_binding_covers_header(agal_lib):
    from agal_b200 import _lib
    bound = {p[0] for p in _lib.PROTOS}
    assert set(declared_functions()) <= bound


def test_params_layout(agal_lib):
    from agal_b200 import _lib
    assert agal_lib.agal_params_size() == C.sizeof(_lib.AgalParams)


def test_defaults_match_parser():
    import agal_b200 as ag
    p = ag.default_params()
    # inc/parser.h:62-138
    assert p.MAX_LEVELS_WALL == 5 and p.MAX_LEVELS_INTERIOR == 4 and p.Nx == 64
    assert p.N_ITER_TOTAL == 640 and p.P_REFINE == 32 and p.N_PROBE_AVE_START == 6400
    assert p.v0 == 1.5625e-5 and p.s6 == 1.98 and p.N_REFINE_START == -3.0
    assert p.I_DIR_NAME == b"../input/" and p.G_FILENAME == b"bunny_ascii.stl"


def test_oracle_defaults_equal_library_defaults():
    """The oracle's restated defaults (used where the CUDA library must not be
    loaded) equal agal_params_default field for field."""
    import agal_b200 as ag
    from agal_b200 import _lib
    from oracle.orc import default_params as orc_default
    a, b = ag.default_params(), orc_default()
    for name, _ in _lib.AgalParams._fields_:
        assert getattr(a, name) == getattr(b, name), name


def test_params_read_nx_factors(tmp_path, capfd):
    import agal_b200 as ag
    (tmp_path / "input.txt").write_text(
        "# comment line\n"
        "N_ITER_TOTAL   100*Nx\n"
        "Nx             32\n"
        "v0             7.8125e-5\n"
        "P_DIR_NAME     ../out/X/\n"
        "NOT_A_KEY      3\n"
        "VOL_I_MAX      1*Nx\n")
    pr = ag.Parser(str(tmp_path))
    assert pr.params_int["Nx"] == 32
    assert pr.params_int["N_ITER_TOTAL"] == 3200   # Nx is read first (parser.h:146-160)
    assert pr.params_int["VOL_I_MAX"] == 32
    assert pr.params_dbl["v0"] == 7.8125e-5
    assert pr.params_str["P_DIR_NAME"] == "../out/X/"
    assert "Invalid input (NOT_A_KEY)" in capfd.readouterr().err


def test_params_errors(tmp_path):
    import agal_b200 as ag
    with pytest.raises(ag.AgalError) as e:
        ag.Parser(str(tmp_path / "missing"))
    assert e.value.code == -6
    (tmp_path / "input.txt").write_text("Nx abc\n")
    with pytest.raises(ag.AgalError) as e:
        ag.Parser(str(tmp_path))
    assert e.value.code == -1


def test_create_rejects_bad_params():
    import agal_b200 as ag
    with pytest.raises(ag.AgalError) as e:
        ag.Case(ag.default_params(Nx=30, n_maxcblocks=1000))
    assert e.value.code == -1
    with pytest.raises(ag.AgalError) as e:
        ag.Case(ag.default_params(velocity_set=7))
    assert e.value.code == -1
