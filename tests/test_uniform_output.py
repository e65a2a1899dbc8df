"""Headless uniform-grid output in the reference's out_direct.dat format
(header: mesh_init.cu:114-150; frames: mesh_print_uniform.cu:96-188).

The restart fixture's run also wrote one frame of the reference's own
out_direct.dat (after M_Advance_PrintData's grid average, interpolation and
refresh).  On the CPU the documented layout and rendering rule are checked on
the reference's bytes against the harness dump of the same state; on the GPU
the library, loaded from the reference's restart.bin of that state, writes
the file again: the header, the time and the level and block fields equal the
reference's byte for byte; rho, u, v are within the cubic-interpolation floor
(the frame's preparation interpolates into ghost cells, and the reference
evaluates its cubic interpolant in FP32 from monomial coefficients, 1e-5..1e-4
from the Lagrange form used here).
"""
import numpy as np
import pytest

from test_oracle import params_for_golden
from test_restart import FIXTURE, fixture

pytestmark = pytest.mark.skipif(not FIXTURE.exists(), reason="restart fixture not generated")


def parse_out_direct(buf: bytes, dims) -> dict:
    nx, ny, nz = dims
    vol = nx * ny * nz
    ip = np.frombuffer(buf, np.int32, 100, 0)
    dp = np.frombuffer(buf, np.float64, 100, 400)
    frames = []
    pos = 1200
    while pos < len(buf):
        t = np.frombuffer(buf, np.float64, 1, pos)[0]
        f = np.frombuffer(buf, np.float64, 6 * vol, pos + 8).reshape(6, nz, ny, nx)
        frames.append((t, f))
        pos += 8 + 48 * vol
    return {"ints": ip, "dbls": dp, "frames": frames, "end": pos}


def render_from_dump(g, dims, print_levels):
    """The rendering rule restated on the harness dump (CPU)."""
    nx, ny, nz = dims
    dim, MC, Q = int(g["dim"]), int(g["MC"]), int(g["Q"])
    blocks = g["blocks"].astype(np.int64)
    row = {int(b): i for i, b in enumerate(blocks)}
    mult = 2 ** (print_levels - 1)
    span = 4 * mult
    out = np.zeros((6, nz, ny, nx))
    out[0] = 1.0
    out[4:] = -1.0
    lvl0 = [i for i in range(len(blocks)) if g["level"][i, 0] == 0]
    fx0 = g["fX"][lvl0]
    step = np.unique(np.round(fx0[:, 0], 6))
    dcb = step[1] - step[0]
    root = {}
    for i in lvl0:
        root[(int(round(g["fX"][i, 0] / dcb)), int(round(g["fX"][i, 1] / dcb)))] = int(blocks[i])
    for Y in range(ny):
        for X in range(nx):
            b = root.get((X // span, Y // span))
            if b is None:
                continue
            px, py, s, L = X % span, Y % span, span, 0
            while L + 1 < print_levels:
                c0 = int(g["nbr_child"][row[b], 0])
                if c0 < 0:
                    break
                h = s // 2
                xi, xj = int(px >= h), int(py >= h)
                b = c0 + xi + 2 * xj
                px, py, s, L = px - xi * h, py - xj * h, h, L + 1
            m = s // 4
            cell = px // m + 4 * (py // m)
            Fm = g["F"][row[b], Q:Q + dim + 1, cell].astype(np.float64)
            out[0, 0, Y, X], out[1, 0, Y, X], out[2, 0, Y, X] = Fm[0], Fm[1], Fm[2]
            out[3, 0, Y, X] = 0.0
            out[4, 0, Y, X], out[5, 0, Y, X] = L, b
    return out


def keys_of(g):
    import json
    return json.loads(str(g["case_keys"]))


def test_reference_frame_layout_and_rendering():
    g = fixture()
    k = keys_of(g)
    pl = int(k["N_PRINT_LEVELS"])
    n = (k["VOL_I_MAX"] - k["VOL_I_MIN"]) * 2 ** (pl - 1)
    dims = (n, n, 1)
    r = parse_out_direct(g["out_direct"].tobytes(), dims)
    assert r["end"] == g["out_direct"].size and len(r["frames"]) == 1
    ip = r["ints"]
    assert ip[0] == (k["N_ITER_TOTAL"] - k["N_OUTPUT_START"]) // k["P_OUTPUT"] and ip[1] == k["P_OUTPUT"]
    assert ip[3] == k["Nx"] and ip[7] == pl and ip[8] == 0
    assert list(ip[9:13]) == [k["VOL_I_MIN"] // 4, k["VOL_I_MAX"] // 4, k["VOL_J_MIN"] // 4, k["VOL_J_MAX"] // 4]
    t, f = r["frames"][0]
    assert t == int(g["steps"]) / k["Nx"]
    ref = render_from_dump(g, dims, pl)
    assert np.array_equal(f, ref)
    assert (f[4] >= 0).all() and set(np.unique(f[4])) <= {0.0, 1.0}


@pytest.mark.gpu
def test_library_writes_the_reference_file(tmp_path):
    import agal_b200 as ag
    g = fixture()
    p, _ = params_for_golden(g)
    p.n_maxcblocks = int(g["n_maxcblocks"])
    src = tmp_path / "restart.bin"
    src.write_bytes(g["restart_bin"].tobytes())
    out = tmp_path / "out_direct.dat"
    with ag.Case(p) as c:
        c.restart_load(src)
        c.uniform_header(out)
        c.uniform_frame(out, int(g["steps"]))
        a, ref = out.read_bytes(), g["out_direct"].tobytes()
        assert len(a) == len(ref)
        assert a[:1200] == ref[:1200]          # header
        dims = c.uniform_dims()
        ta, fa = parse_out_direct(a, dims)["frames"][0]
        tr, fr = parse_out_direct(ref, dims)["frames"][0]
        assert ta == tr
        for i in (3, 4, 5):                    # w (0 in 2D), level, block ID
            assert np.array_equal(fa[i], fr[i]), i
        assert np.abs(fa[:3] - fr[:3]).max() < 1e-4
        assert (fa[:3] == fr[:3]).mean() > 0.9
