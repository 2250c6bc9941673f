"""8th-order FD operator ("Order of FD Operator" : "8") on the CPU restatement.

The reference parses this key and runs its step only for 4
(src/src_cpu/cpumodelling.cpp:121, `if (NJ == 4)`), so there is no reference
output; the operator is checked on what an 8th-order operator must do:
  * at a coarse spacing its traces stay close to a twice-finer solution where
    the 4th-order operator's are visibly dispersed (homogeneous medium, the
    window closing before any boundary reflection arrives);
  * FP32 agrees with FP64;
  * order 4 is untouched (the golden tests pin it to the reference binary);
  * the adjoint oracle refuses it.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _homogeneous_run(n, d, nb, order, precision=O.F64):
    L, omax = 2400.0, 1000.0
    p = O.Params(n, n, nb, d, d, 0.6, 0.001, 0.002, 20.0, 0, order)
    vp = np.full((n, n), 2000.0, np.float32)
    rho = np.full((n, n), 1000.0, np.float32)
    rx = np.arange(L / 2 + 300, L / 2 + omax, 20, dtype=np.float32)
    return O.forward(p, vp, rho, (L / 2, L / 2), rx, np.full(rx.size, L / 2, np.float32), precision=precision)


def test_order8_is_less_dispersive_than_order4():
    """10 m cells at 20 Hz (about 4 cells per shortest wavelength): against the
    8th-order solution on 5 m cells, order 4 is ~22% off, order 8 ~1.4%."""
    coarse4 = _homogeneous_run(240, 10.0, 20, 4)
    coarse8 = _homogeneous_run(240, 10.0, 20, 8)
    fine8 = _homogeneous_run(480, 5.0, 40, 8)
    e4, e8 = O.rel_l2(coarse4, fine8), O.rel_l2(coarse8, fine8)
    assert e8 <= 0.03, e8
    assert e4 >= 5 * e8, (e4, e8)


def test_order8_fp32_matches_fp64():
    nx, nz = 90, 70
    rng = np.random.default_rng(8)
    vp = (1800 + 900 * rng.random((nx, nz))).astype(np.float32)
    rho = (1500 + 400 * rng.random((nx, nz))).astype(np.float32)
    p = O.Params(nx, nz, 30, 10.0, 10.0, 0.3, 0.001, 0.002, 18.0, 0, 8)
    rx = np.arange(1, nx - 1) * 10.0
    a = O.forward(p, vp, rho, (450.0, 100.0), rx, np.full(rx.size, 20.0), precision=O.F64)
    b = O.forward(p, vp, rho, (450.0, 100.0), rx, np.full(rx.size, 20.0), precision=O.F32)
    assert O.rel_l2(b, a) <= 1e-6


def test_order8_differs_from_order4_and_small_grids_run():
    """Grids narrower than the 8-tap stencil fall back to the reference's rows
    everywhere; a 3 x 3 model with a 2-cell sponge still runs."""
    nx, nz = 3, 3
    vp = np.full((nx, nz), 2000.0, np.float32)
    rho = np.full((nx, nz), 1000.0, np.float32)
    for order in (4, 8):
        p = O.Params(nx, nz, 2, 10.0, 10.0, 0.02, 0.001, 0.001, 30.0, 0, order)
        s = O.forward(p, vp, rho, (10.0, 10.0), [0.0, 20.0], [10.0, 10.0])
        assert np.all(np.isfinite(s)) and np.abs(s).max() > 0
    nx, nz = 60, 40
    rng = np.random.default_rng(2)
    vp = (2000 + 300 * rng.random((nx, nz))).astype(np.float32)
    rho = np.full((nx, nz), 1200.0, np.float32)
    out = {}
    for order in (4, 8):
        p = O.Params(nx, nz, 20, 10.0, 10.0, 0.2, 0.001, 0.001, 20.0, 0, order)
        out[order] = O.forward(p, vp, rho, (300.0, 50.0), np.arange(nx) * 10.0, np.full(nx, 30.0))
    assert O.rel_l2(out[8], out[4]) > 1e-3


def test_gradient_oracle_refuses_order8():
    nx, nz = 20, 20
    vp = np.full((nx, nz), 2000.0, np.float32)
    rho = np.full((nx, nz), 1000.0, np.float32)
    p = O.Params(nx, nz, 10, 10.0, 10.0, 0.05, 0.001, 0.001, 25.0, 0, 8)
    with pytest.raises(ValueError):
        O.gradient(p, vp, rho, (100.0, 50.0), [50.0], [50.0], None)
