"""The adjoint kernels add the receiver adjoint source only in strips whose rows
hold receivers (the forward records only there): on a grid three strips tall,
with receivers down a borehole confined to the middle strip, or spread over all
three, the FP32 gradient stays within the bar of the FP64 discrete adjoint
(oracle/s2d_oracle.c) for the 4th- and the 8th-order operator."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NX, NZ, NB, D = 40, 260, 32, 10.0
GRAD_TOL = 1e-4   # rel-L2 of the FP32 gradient field against the FP64 adjoint


def _model(seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(0, 1, NX)[:, None]
    z = np.linspace(0, 1, NZ)[None, :]
    vp = 1800 + 900 * z + 80 * np.sin(6 * x) * np.cos(5 * z) + 20 * rng.standard_normal((NX, NZ))
    rho = 1300 + 600 * z + 40 * np.cos(4 * x + 3 * z)
    return vp.astype(np.float32), rho.astype(np.float32)


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


# receiver depths (grid cells): padded rows 152..197 lie in the second strip
# of both strip layouts (120 output rows for order 4, 112 for order 8);
# 2..255 cross all three
GEOMS = {"middle_strip": np.arange(120, 166, 3), "all_strips": np.arange(2, 256, 9)}


@pytest.mark.parametrize("order", [4, 8])
@pytest.mark.parametrize("geom", sorted(GEOMS))
def test_borehole_receivers_match_fp64_adjoint(ctx, order, geom):
    from seis2d_b200 import Shot, Wave
    T = 0.3 if order == 4 else 0.15
    vp, rho = _model(41 + order)
    iz = GEOMS[geom]
    rec = np.stack([np.full(iz.size, 25 * D), iz * D], 1).astype(np.float32)
    src = (12 * D, 140 * D)
    p = O.Params(NX, NZ, NB, D, D, T, 0.001, 0.002, 20.0, 0, order)
    nt = O.derive(p)["real_nt"]
    adj = np.random.default_rng(53).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB, fd_order=order)
    wave = Wave(T, 0.001, 0.002, 20.0)
    try:
        g = ctx.gradient([Shot(m, src, rec)], wave, adj)
        if order == 4:
            # the adjoint with plain loads (the default feeds it by
            # asynchronous copies): the same bits
            ctx.set_option("adjoint_blocks", 3)
            try:
                g13 = ctx.gradient([Shot(m, src, rec)], wave, adj)
            finally:
                ctx.set_option("adjoint_blocks", 13)
            np.testing.assert_array_equal(g13.grad_vp, g.grad_vp)
            np.testing.assert_array_equal(g13.grad_rho, g.grad_rho)
    finally:
        m.release()
    ref = O.gradient(p, vp, rho, src, rec[:, 0], rec[:, 1], adj.astype(np.float64))
    e_vp = O.rel_l2(g.grad_vp, ref["grad_vp"])
    e_rho = O.rel_l2(g.grad_rho, ref["grad_rho"])
    assert e_vp <= GRAD_TOL and e_rho <= GRAD_TOL, (e_vp, e_rho)
