"""8th-order FD operator ("Order of FD Operator" : "8") on the CPU restatement.

The reference parses this key and runs its step only for 4
(src/src_cpu/cpumodelling.cpp:121, `if (NJ == 4)`), so there is no reference
output; the operator is checked on what an 8th-order operator must do:
  * at a coarse spacing its traces stay close to a twice-finer solution where
    the 4th-order operator's are visibly dispersed (homogeneous medium, the
    window closing before any boundary reflection arrives);
  * FP32 agrees with FP64;
  * order 4 is untouched (the golden tests pin it to the reference binary);
  * its FP64 adjoint passes the dot-product test and central differences.
"""
import numpy as np

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


NX, NZ, NB = 40, 30, 12
P8 = O.Params(NX, NZ, NB, 10.0, 10.0, 0.15, 0.001, 0.002, 25.0, 0, 8)
SRC = (200.0, 50.0)
RX = np.arange(2, 38, 3) * 10.0
RZ = np.full(RX.size, 20.0)


def _model():
    rng = np.random.default_rng(1)
    vp = (2000 + 300 * rng.random((NX, NZ))).astype(np.float32)
    rho = (1500 + 200 * rng.random((NX, NZ))).astype(np.float32)
    return vp, rho


def test_order8_adjoint_forward_is_the_order8_forward():
    vp, rho = _model()
    g = O.gradient(P8, vp, rho, SRC, RX, RZ, None)["seis64"]
    f = O.forward(P8, vp, rho, SRC, RX, RZ, precision=O.F64)
    assert O.rel_l2(f, g) <= 1e-7


def test_order8_adjoint_dot_product():
    vp, rho = _model()
    d = O.derive(P8)
    rng = np.random.default_rng(2)
    w = rng.standard_normal(d["nts"] + 1)
    r = rng.standard_normal((RX.size, d["real_nt"]))
    g = O.gradient(P8, vp, rho, SRC, RX, RZ, r, wavelet=w)
    traces = O.gradient(P8, vp, rho, SRC, RX, RZ, None, wavelet=w)["seis64"]
    ix, iz = int(SRC[0] * np.float32(0.1)), int(SRC[1] * np.float32(0.1))
    coef = float(np.float32(0.001)) * (float(vp[ix, iz]) ** 2 * float(rho[ix, iz])) / float(np.float32(100.0))
    n = min(d["nts"] + 1, d["fd_nt"])
    lhs = np.sum(traces * r)
    rhs = np.sum(w[:n] * coef * g["src_adj"][:n])
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_order8_adjoint_finite_differences():
    """Cells inside, next to the sponge (where the operator falls back to the
    reference's rows) and on the edges of the model."""
    vp, rho = _model()
    base = O.gradient(P8, vp, rho, SRC, RX, RZ, None)["seis64"]
    dobs = 0.9 * base + 0.01 * np.random.default_rng(3).standard_normal(base.shape)

    def J(v, r):
        s = O.gradient(P8, v, r, SRC, RX, RZ, None)["seis64"]
        return 0.5 * np.sum((s - dobs) ** 2)

    G = O.gradient(P8, vp, rho, SRC, RX, RZ, base - dobs)
    for i, j in [(5, 5), (20, 15), (0, 0), (20, 5), (20, 2), (39, 10), (20, 29)]:
        for name, arr, grad in (("vp", vp, G["grad_vp"]), ("rho", rho, G["grad_rho"])):
            scale = np.abs(grad).max()
            eps = float(arr[i, j]) * 1e-3
            a1, a2 = arr.copy(), arr.copy()
            a1[i, j] += eps
            a2[i, j] -= eps
            jp = J(a1, rho) if name == "vp" else J(vp, a1)
            jm = J(a2, rho) if name == "vp" else J(vp, a2)
            fd = (jp - jm) / (float(a1[i, j]) - float(a2[i, j]))
            assert abs(fd - grad[i, j]) <= 1e-5 * scale + 2e-4 * abs(fd), (name, i, j, fd, grad[i, j], scale)
