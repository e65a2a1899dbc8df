"""agal_mass_momentum_noalloc (static device scratch, allocates nothing)
against agal_mass_momentum (context-owned cudaMalloc'd scratch).

Both launch the same FP64 partial-sum kernels in the same order, so the
results agree to rounding: held here to 1e-13 relative (mass) and 1e-12
absolute (momentum), on two calls in a row after stepping.  Collected last
so that it also runs after every other GPU test has used the device."""
import numpy as np
import pytest

import agal_b200 as ag
from agal_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-13, 1e-12


def _case(Q, N, storage, **extra):
    dim = 2 if Q == 9 else 3
    kw = dict(velocity_set={9: _lib.D2Q9, 19: _lib.D3Q19, 27: _lib.D3Q27}[Q], Nx=N,
              MAX_LEVELS_WALL=1, MAX_LEVELS_INTERIOR=1, v0=5e-4,
              bc_preset=_lib.BC_LDC2D if dim == 2 else _lib.BC_LDC3D, storage=storage,
              n_maxcblocks=(N // 4) ** dim + 5)
    kw.update(extra)
    return ag.default_params(**kw)


@pytest.mark.parametrize("Q,N,storage", [(9, 64, _lib.STORE_FP32), (9, 256, _lib.STORE_FP64),
                                         (19, 32, _lib.STORE_FP16), (27, 16, _lib.STORE_FP32)])
def test_noalloc_matches_mass_momentum(Q, N, storage):
    p = _case(Q, N, storage)
    with ag.Case(p) as c:
        c.set_ic(0)
        for steps in (0, 37, 50):
            c.advance_n(steps, use_graph=False) if steps else None
            ref = c.mass_momentum()
            a = c.mass_momentum_noalloc()
            b = c.mass_momentum_noalloc()
            assert a.shape == ref.shape
            assert abs(a[0] - ref[0]) <= RTOL * abs(ref[0])
            assert np.abs(a[1:] - ref[1:]).max() <= ATOL
            assert abs(b[0] - ref[0]) <= RTOL * abs(ref[0])
            assert np.abs(b[1:] - ref[1:]).max() <= ATOL


def test_noalloc_two_contexts_in_turn():
    """Two contexts on one device share the static scratch; calls made one
    after the other each see their own sums."""
    p1 = _case(9, 64, _lib.STORE_FP32)
    p2 = _case(9, 64, _lib.STORE_FP32, ic_preset=_lib.IC_UNIFORM, u_ref=0.02)
    with ag.Case(p1) as c1, ag.Case(p2) as c2:
        c1.set_ic(0)
        c2.set_ic(0)
        c1.advance_n(20, use_graph=False)
        c2.advance_n(20, use_graph=False)
        for c in (c1, c2, c1, c2):
            ref = c.mass_momentum()
            a = c.mass_momentum_noalloc()
            assert abs(a[0] - ref[0]) <= RTOL * abs(ref[0])
            assert np.abs(a[1:] - ref[1:]).max() <= ATOL


def test_noalloc_rejects_more_partials_than_the_scratch_holds():
    """8192 x 8196 cells need 262,272 partials (> 262,144): rejected with
    AGAL_ERR_PARAM before any launch; the allocating entry point still works."""
    p = _case(9, 8192, _lib.STORE_FP16, L_fy=8196.0 / 8192.0, bc_preset=_lib.BC_NONE,
              ic_preset=_lib.IC_REST, n_maxcblocks=2048 * 2049 + 5)
    with ag.Case(p) as c:
        c.set_ic(0)
        with pytest.raises(ag.AgalError) as e:
            c.mass_momentum_noalloc()
        assert e.value.code == _lib.ERR_PARAM
        assert "static scratch" in str(e.value)
        m = c.mass_momentum()
        assert abs(m[0] - 8192.0 * 8196.0) < 1e-6 * 8192.0 * 8196.0


def test_noalloc_allocates_no_device_memory():
    """On a fresh context whose mesh needs the largest scratch the entry point
    accepts (8192^2 cells: 262,144 partials of 4 doubles, 8 MiB), repeated
    noalloc calls leave the device's free memory (cudaMemGetInfo) unchanged;
    the allocating entry point on the same context grows its own scratch."""
    import torch
    p = _case(9, 8192, _lib.STORE_FP16, bc_preset=_lib.BC_NONE, ic_preset=_lib.IC_REST,
              n_maxcblocks=2048 * 2048 + 5)
    torch.cuda.mem_get_info(0)
    with ag.Case(p) as c:
        c.set_ic(0)
        c.sync()
        free0, _ = torch.cuda.mem_get_info(0)
        for _ in range(3):
            a = c.mass_momentum_noalloc()
        c.sync()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, (free0, free1)
        assert abs(a[0] - 8192.0 * 8192.0) < 1e-6 * 8192.0 * 8192.0
        m = c.mass_momentum()
        c.sync()
        free2, _ = torch.cuda.mem_get_info(0)
        assert free2 < free1, (free1, free2)
        assert abs(m[0] - a[0]) <= RTOL * abs(m[0])
