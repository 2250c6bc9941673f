"""Edge cases of the CUDA forward path against the oracle: grids narrower than
the stencils (down to one physical cell), a shot without receivers inside a
batch, and a grid beyond the library's addressing limit (refused before any
allocation)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5   # seismogram rel-L2, FP32 CUDA vs the FP64 oracle


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("nx,nz,nb,order", [(1, 1, 2, 4), (1, 1, 2, 8), (2, 300, 3, 4), (300, 1, 5, 8),
                                            (3, 2, 4, 4), (7, 9, 2, 8), (130, 2, 2, 4)])
def test_tiny_grids_match_oracle(ctx, nx, nz, nb, order):
    from seis2d_b200 import Shot, Wave
    rng = np.random.default_rng(nx * 1000 + nz)
    vp = (2000 + 200 * rng.random((nx, nz))).astype(np.float32)
    rho = (1500 + 100 * rng.random((nx, nz))).astype(np.float32)
    rec = np.stack([np.arange(nx) * 10.0, np.zeros(nx)], 1).astype(np.float32)
    m = ctx.model(vp, rho, 10.0, 10.0, nb, fd_order=order)
    got = ctx.forward([Shot(m, (0.0, 0.0), rec)], Wave(0.05, 0.001, 0.001, 25.0))[0]
    p = O.Params(nx, nz, nb, 10.0, 10.0, 0.05, 0.001, 0.001, 25.0, 0, order)
    ref = O.forward(p, vp, rho, (0.0, 0.0), rec[:, 0], rec[:, 1], O.F64)
    assert np.abs(ref).max() > 0
    assert O.rel_l2(got, ref) <= TOL
    m.release()


def test_shot_without_receivers_in_a_batch(ctx):
    from seis2d_b200 import Shot, Wave
    nx, nz = 80, 60
    rng = np.random.default_rng(3)
    vp = (1800 + 600 * rng.random((nx, nz))).astype(np.float32)
    rho = np.full((nx, nz), 1400.0, np.float32)
    m = ctx.model(vp, rho, 10.0, 10.0, 20)
    rec = np.stack([np.arange(nx) * 10.0, np.full(nx, 20.0)], 1).astype(np.float32)
    none = np.zeros((0, 2), np.float32)
    w = Wave(0.2, 0.001, 0.002, 20.0)
    batch = ctx.forward([Shot(m, (200.0, 20.0), rec), Shot(m, (400.0, 20.0), none), Shot(m, (600.0, 20.0), rec)], w)
    assert batch[1].shape == (0, batch[0].shape[1])
    for src, got in (((200.0, 20.0), batch[0]), ((600.0, 20.0), batch[2])):
        alone = ctx.forward([Shot(m, src, rec)], w)[0]
        np.testing.assert_array_equal(got, alone)
    m.release()


def test_grid_beyond_the_addressing_limit_is_refused():
    """8 state fields of a 17000 x 17000 grid exceed 2^31 elements: the model
    is refused with S2D_ERR_ARG before any copy or allocation (the buffers
    passed are a few bytes; the library must not read them)."""
    from seis2d_b200 import Context
    from seis2d_b200 import _lib as L
    c = Context(0)
    try:
        tiny = np.zeros(4, np.float32)
        mid = C.c_int(-1)
        rc = L.lib().s2d_model_create(c._h, 17000, 17000, 5.0, 5.0, 60, C.c_void_p(tiny.ctypes.data),
                                      C.c_void_p(tiny.ctypes.data), 0, C.byref(mid))
        assert rc == L.S2D_ERR_ARG and mid.value == -1
        assert b"too large" in L.lib().s2d_last_error(c._h)
    finally:
        c.close()


def test_grid_wider_than_the_launch_limit_is_refused():
    """A padded grid of more than 65535 columns (70000 x 4 cells, whose state
    is well inside the addressing limit) is refused with S2D_ERR_ARG and a
    message naming the limit, before any copy or allocation."""
    from seis2d_b200 import Context
    from seis2d_b200 import _lib as L
    c = Context(0)
    try:
        tiny = np.zeros(4, np.float32)
        mid = C.c_int(-1)
        rc = L.lib().s2d_model_create(c._h, 70000, 4, 5.0, 5.0, 60, C.c_void_p(tiny.ctypes.data),
                                      C.c_void_p(tiny.ctypes.data), 0, C.byref(mid))
        assert rc == L.S2D_ERR_ARG and mid.value == -1
        assert b"65535" in L.lib().s2d_last_error(c._h)
    finally:
        c.close()
