"""External flow in a channel (the D3Q27 icosphere channel of the benchmark
configurations, reduced): a box of 1 x 0.5 x 0.5 instead of the unit cube.

The reference indexes face bins and voxelizer cells as coordinate x density
and coordinate x N, which only agrees with its own bin sizes on the unit
cube; this library indexes per axis (bins per unit length), which is the
same arithmetic on the unit cube and consistent on a channel.  Checked here:
the sphere voxelizes to the same solid cells in the channel as in the cube,
the CUDA chain equals the FP64 oracle bit for bit in its integer arrays, and
FP16 / FP32 drag and lift stay within 1% of the FP64 run."""
import numpy as np
import pytest

import agal_b200 as ag
from agal_b200 import _lib
from agal_b200.geometry import icosphere

pytestmark = pytest.mark.gpu

NX = 64
CENTRE = (0.25, 0.25, 0.25)
RADIUS = 4.0 / NX            # diameter 8 root cells


def channel_params(storage=_lib.STORE_FP32, cube=False, levels=3, **kw):
    d = dict(velocity_set=_lib.D3Q27, Nx=NX, L_fy=1.0 if cube else 0.5, L_fz=1.0 if cube else 0.5,
             MAX_LEVELS_WALL=levels, MAX_LEVELS_INTERIOR=1, v0=0.05 * 2 * RADIUS / 200.0, P_REFINE=10 ** 8,
             G_BIN_DENSITY=8, G_BIN_LEVELS=levels, G_BIN_SPEC=2, G_BIN_MAKE_LINKS=1, G_NEAR_WALL_DISTANCE=0.03,
             S_BC_TYPE=1, S_FORCE_TYPE=0, S_FORCE_ORDER=2, bc_preset=_lib.BC_FPSC3D, ic_preset=_lib.IC_UNIFORM,
             u_ref=0.05, ic_noise=0.01, seed=7, storage=storage,
             n_maxcblocks=(NX // 4) ** 3 + 6000)
    d.update(kw)
    return ag.default_params(**d)


def sphere_faces(subdiv=4):
    return icosphere(subdiv, RADIUS, CENTRE, seed=3)


def solid_centres(c, p, L=None):
    """Centres of the solid cells of level L (default: the finest), in
    domain units, and the level's cell size."""
    nmb = p.n_maxcblocks
    cnt = c.counts()
    L = cnt["max_levels"] - 1 if L is None else L
    ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)[L, : cnt["n_ids"][L]].astype(np.int64)
    cm = c.dump(_lib.ARR_CELLS_ID_MASK).reshape(nmb, 64)[ids]
    fX = c.dump(_lib.ARR_CBLOCK_F_X).reshape(3, nmb)[:, ids].T
    dx = (1.0 / NX) / 2 ** L
    t = np.arange(64)
    off = np.stack([t % 4, (t // 4) % 4, t // 16], axis=1) * dx + 0.5 * dx
    pts = fX[:, None, :] + off[None, :, :]
    return pts[cm == -1], dx


def solid_volume(c, p):
    """Volume of the solid cells of the leaf blocks (blocks without children)
    over all levels."""
    nmb = p.n_maxcblocks
    cnt = c.counts()
    child = c.dump(_lib.ARR_CBLOCK_ID_NBR_CHILD).reshape(-1, nmb)[0]
    ids_all = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
    cm = c.dump(_lib.ARR_CELLS_ID_MASK).reshape(nmb, 64)
    vol = 0.0
    for L in range(cnt["max_levels"]):
        ids = ids_all[L, : cnt["n_ids"][L]].astype(np.int64)
        leaf = ids[child[ids] < 0]
        vol += float((cm[leaf] == -1).sum()) * ((1.0 / NX) / 2 ** L) ** 3
    return vol


def test_channel_voxelizes_like_the_cube():
    out = {}
    for cube in (True, False):
        p = channel_params(cube=cube)
        with ag.Case(p) as c:
            c.set_geometry(sphere_faces())
            c.set_ic(0)
            c.refine_near_wall()
            pts, dx = solid_centres(c, p)
            out[cube] = np.round(pts / dx).astype(np.int64)
            if not cube:
                vol = solid_volume(c, p)
                coarse, dx0 = solid_centres(c, p, 0)
    a = {tuple(r) for r in out[True]}
    b = {tuple(r) for r in out[False]}
    assert a == b and len(a) > 0
    # the solid leaf cells fill the sphere, centred on it
    sphere = 4.0 / 3.0 * np.pi * RADIUS ** 3
    assert abs(vol - sphere) < 0.06 * sphere, (vol, sphere)
    assert np.abs(coarse.mean(axis=0) - np.asarray(CENTRE)).max() < dx0


def test_channel_fp64_matches_oracle():
    from oracle.orc import OracleCase
    p = channel_params(storage=_lib.STORE_FP64)
    steps = 6
    f = sphere_faces(3)
    with ag.Case(p) as c:
        c.set_geometry(f)
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(steps, use_graph=False)
        c.sync()
        o = OracleCase(p, p.n_maxcblocks, fp64=True)
        o.set_geometry(f)
        o.set_ic(0)
        o.refine_near_wall()
        o.advance_n(steps)
        for k in (_lib.ARR_CELLS_ID_MASK, _lib.ARR_CBLOCK_ID_MASK, _lib.ARR_CBLOCK_ID_NBR, _lib.ARR_CBLOCK_ID_REF,
                  _lib.ARR_CBLOCK_LEVEL, _lib.ARR_CBLOCK_ID_ONB_SOLID, _lib.ARR_CELLS_F_X_B):
            assert np.array_equal(c.dump(k), o.dump(k)), k
        nmb = p.n_maxcblocks
        cnt = c.counts()
        ids = c.dump(_lib.ARR_ID_SET).reshape(-1, nmb)
        blocks = np.sort(np.concatenate([ids[L, : cnt["n_ids"][L]] for L in range(cnt["max_levels"])]))
        Fc = c.dump(_lib.ARR_F).reshape(27, nmb, 64)[:, blocks]
        Fo = o.dump(_lib.ARR_F).reshape(27, nmb, 64)[:, blocks]
        assert np.abs(Fc - Fo).max() < 1e-11


def drag_lift(storage, steps):
    p = channel_params(storage=storage)
    with ag.Case(p) as c:
        c.set_geometry(sphere_faces())
        c.set_ic(0)
        c.refine_near_wall()
        c.advance_n(steps - 1, use_graph=True)
        c.forces()                       # reset the partials
        c.advance_n(1, use_graph=True)
        fr = c.forces()
    return np.array([fr[0] - fr[1], fr[2] - fr[3], fr[4] - fr[5]])


def test_channel_half_storage_drag_lift_within_one_percent():
    steps = 400
    f64 = drag_lift(_lib.STORE_FP64, steps)
    assert abs(f64[0]) > 10 * np.abs(f64[1:]).max()   # the drag dominates
    for st in (_lib.STORE_FP32, _lib.STORE_FP16):
        f = drag_lift(st, steps)
        print(st, f, f64)
        assert abs(f[0] - f64[0]) < 0.01 * abs(f64[0]), (st, f, f64)
        assert np.abs(f[1:] - f64[1:]).max() < 0.01 * abs(f64[0]), (st, f, f64)
