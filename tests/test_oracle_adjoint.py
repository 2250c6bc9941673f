"""The FP64 CPU adjoint (oracle/s2d_oracle.c: orc_gradient), which the CUDA
gradient is checked against, checked on its own: the dot-product test of the
source-to-traces map and central finite differences of the FP64 misfit."""
import numpy as np

from oracle import oracle as O

NX, NZ, NB = 40, 30, 32
P = O.Params(NX, NZ, NB, 10.0, 10.0, 0.15, 0.001, 0.002, 25.0)
SRC = (200.0, 50.0)
RX = np.arange(2, 38, 3) * 10.0
RZ = np.full(RX.size, 20.0)


def _model():
    rng = np.random.default_rng(1)
    vp = (2000 + 300 * rng.random((NX, NZ))).astype(np.float32)
    rho = (1500 + 200 * rng.random((NX, NZ))).astype(np.float32)
    return vp, rho


def test_fp64_adjoint_dot_product():
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


def test_fp64_adjoint_finite_differences():
    vp, rho = _model()
    base = O.gradient(P, vp, rho, SRC, RX, RZ, None)["seis64"]
    dobs = 0.9 * base + 0.01 * np.random.default_rng(3).standard_normal(base.shape)

    def J(v, r):
        s = O.gradient(P, v, r, SRC, RX, RZ, None)["seis64"]
        return 0.5 * np.sum((s - dobs) ** 2)

    G = O.gradient(P, vp, rho, SRC, RX, RZ, base - dobs)
    for i, j in [(5, 5), (20, 15), (0, 0), (20, 5), (20, 2), (39, 10)]:
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


def test_checkpoints_and_threads_keep_the_bits():
    """Checkpointed recompute (any segment length) and the threaded loops
    give the same FP64 gradient, traces and source adjoint bit for bit, for
    the 4th- and the 8th-order operator; the forward alone gives the same
    traces."""
    vp, rho = _model()
    d = O.derive(P)
    r = np.random.default_rng(3).standard_normal((RX.size, d["real_nt"]))
    keys = ("grad_vp", "grad_rho", "grad_kappa", "grad_bx", "grad_bz", "src_adj", "seis64")
    for order in (4, 8):
        p = O.Params(NX, NZ, NB, 10.0, 10.0, 0.15, 0.001, 0.002, 25.0, 0, order)
        whole = O.gradient(p, vp, rho, SRC, RX, RZ, r)
        try:
            for seg, threads in ((37, 1), (1, 1), (0, 4), (37, 3)):
                O.set_threads(threads)
                got = O.gradient(p, vp, rho, SRC, RX, RZ, r, segment=seg)
                for k in keys:
                    np.testing.assert_array_equal(got[k], whole[k], err_msg=f"order {order} {k} {seg} {threads}")
        finally:
            O.set_threads(1)
        fwd = O.gradient(p, vp, rho, SRC, RX, RZ, None, segment=37)
        np.testing.assert_array_equal(fwd["seis64"], whole["seis64"])
        assert not fwd["grad_vp"].any() and not fwd["src_adj"].any()
