"""Free surface ("Free surface" : "1") on the CPU restatement.

The reference parses this job-card key and ignores it
(src/src_cpu/json_parser.cpp:236-244; its Instructions: "Free surface yet not
implemented"), so there is no reference output to match.  The rule here is the
vacuum form of a pressure-release surface at the first model row: kappa = 0
on padded rows 0..nb.  It is checked on physics instead:
  * pressure is exactly zero on the surface row and above it, at every step;
  * in a homogeneous medium the traces equal, to the accuracy of the scheme,
    the image-source solution: the same run without a surface on a deeper grid,
    with the source and an opposite-sign source mirrored across the surface row;
  * a source on the surface injects nothing;
  * the FP64 adjoint stays exact (dot-product test, central differences), with
    kappa on the vacuum rows held fixed.
"""
import numpy as np

from oracle import oracle as O

D = 10.0


def _homogeneous(nx, nz):
    return np.full((nx, nz), 2000.0, np.float32), np.full((nx, nz), 1000.0, np.float32)


def test_pressure_is_zero_on_and_above_the_surface():
    nx, nz, nb = 60, 40, 32
    p = O.Params(nx, nz, nb, D, D, 0.2, 0.001, 0.001, 20.0, 1)
    vp, rho = _homogeneous(nx, nz)
    vp[:, 20:] = 2600.0
    rx = np.arange(0, nx) * D
    for prec in (O.F64, O.F32):
        seis, (px, pz, vx, vz, pp) = O.forward(p, vp, rho, (300.0, 50.0), rx, np.full(nx, 0.0),
                                               precision=prec, kt_stop=150, want_state=True)
        assert np.all(px[:, :nb + 1] == 0) and np.all(pz[:, :nb + 1] == 0) and np.all(pp[:, :nb + 1] == 0)
        assert np.abs(pp[:, nb + 1:]).max() > 0
        # receivers on the surface row record zero
        assert np.all(seis == 0)


def test_traces_match_the_image_source_solution():
    nx, nz, M, ks, kr = 200, 120, 60, 10, 6
    rx = np.arange(nx) * D

    def run(nzz, fs, zsrc, zrec):
        p = O.Params(nx, nzz, 32, D, D, 0.5, 0.001, 0.001, 15.0, fs)
        vp, rho = _homogeneous(nx, nzz)
        return O.forward(p, vp, rho, (1000.0, zsrc * D), rx, np.full(nx, zrec * D, np.float32)).astype(np.float64)

    with_surface = run(nz, 1, ks, kr)
    without = run(nz, 0, ks, kr)
    # surface at row M of a deeper grid: source at M + ks, image at M - ks
    image = run(nz + M, 0, M + ks, M + kr) - run(nz + M, 0, M - ks, M + kr)
    assert O.rel_l2(with_surface, image) <= 0.06
    # the surface ghost is what the check sees
    assert O.rel_l2(without, image) >= 0.5


def test_source_on_the_surface_injects_nothing():
    nx, nz = 50, 30
    p = O.Params(nx, nz, 32, D, D, 0.15, 0.001, 0.001, 20.0, 1)
    vp, rho = _homogeneous(nx, nz)
    rx = np.arange(nx) * D
    seis = O.forward(p, vp, rho, (250.0, 0.0), rx, np.full(nx, 50.0))
    assert np.all(seis == 0)
    p0 = O.Params(nx, nz, 32, D, D, 0.15, 0.001, 0.001, 20.0, 0)
    assert np.abs(O.forward(p0, vp, rho, (250.0, 0.0), rx, np.full(nx, 50.0))).max() > 0


def test_fp32_matches_fp64_with_the_surface():
    nx, nz = 80, 50
    p = O.Params(nx, nz, 40, D, D, 0.3, 0.001, 0.002, 18.0, 1)
    rng = np.random.default_rng(4)
    vp = (2000 + 500 * rng.random((nx, nz))).astype(np.float32)
    rho = (1600 + 300 * rng.random((nx, nz))).astype(np.float32)
    rx = np.arange(1, nx - 1) * D
    a = O.forward(p, vp, rho, (400.0, 30.0), rx, np.full(rx.size, 20.0), precision=O.F64)
    b = O.forward(p, vp, rho, (400.0, 30.0), rx, np.full(rx.size, 20.0), precision=O.F32)
    assert O.rel_l2(b, a) <= 1e-6


NX, NZ, NB = 40, 30, 32
P = O.Params(NX, NZ, NB, 10.0, 10.0, 0.15, 0.001, 0.002, 25.0, 1)
SRC = (200.0, 30.0)
RX = np.arange(2, 38, 3) * 10.0
RZ = np.full(RX.size, 20.0)


def _model():
    rng = np.random.default_rng(1)
    vp = (2000 + 300 * rng.random((NX, NZ))).astype(np.float32)
    rho = (1500 + 200 * rng.random((NX, NZ))).astype(np.float32)
    return vp, rho


def test_fp64_adjoint_dot_product_with_the_surface():
    vp, rho = _model()
    d = O.derive(P)
    rng = np.random.default_rng(2)
    w = rng.standard_normal(d["nts"] + 1)
    r = rng.standard_normal((RX.size, d["real_nt"]))
    g = O.gradient(P, vp, rho, SRC, RX, RZ, r, wavelet=w)
    traces = O.gradient(P, vp, rho, SRC, RX, RZ, None, wavelet=w)["seis64"]
    ix, iz = int(SRC[0] * np.float32(0.1)), int(SRC[1] * np.float32(0.1))
    coef = float(np.float32(0.001)) * (float(vp[ix, iz]) ** 2 * float(rho[ix, iz])) / float(np.float32(100.0))
    n = min(d["nts"] + 1, d["fd_nt"])
    lhs = np.sum(traces * r)
    rhs = np.sum(w[:n] * coef * g["src_adj"][:n])
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_fp64_adjoint_finite_differences_with_the_surface():
    """Cells on the surface row included: vp there only sets kappa on rows the
    surface holds at 0, so its exact derivative is 0; rho there still enters
    through the buoyancy."""
    vp, rho = _model()
    base = O.gradient(P, vp, rho, SRC, RX, RZ, None)["seis64"]
    dobs = 0.9 * base + 0.01 * np.random.default_rng(3).standard_normal(base.shape)

    def J(v, r):
        s = O.gradient(P, v, r, SRC, RX, RZ, None)["seis64"]
        return 0.5 * np.sum((s - dobs) ** 2)

    G = O.gradient(P, vp, rho, SRC, RX, RZ, base - dobs)
    assert np.all(G["grad_vp"][:, 0] == 0)
    assert np.abs(G["grad_rho"][:, 0]).max() > 0
    for i, j in [(5, 5), (20, 15), (20, 0), (20, 1), (20, 3), (39, 10)]:
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
