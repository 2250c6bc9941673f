"""8th-order operator (S2D_MODEL_ORDER8, job card "Order of FD Operator" : "8")
on the GPU, against the CPU restatement of the same operator (its physics is
checked in tests/test_oracle_order8.py).

The reference parses the key and steps only for 4 (src/src_cpu/
cpumodelling.cpp:121), so there is no reference output; the oracle is the bar
at the tolerance of the reference-parity tests.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5   # seismogram rel-L2, FP32 CUDA vs the FP64 oracle
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _model(nx, nz, seed):
    rng = np.random.default_rng(seed)
    x = np.linspace(0, 1, nx)[:, None]
    z = np.linspace(0, 1, nz)[None, :]
    vp = 1800 + 1200 * z + 150 * np.sin(7 * x) * np.cos(4 * z) + 25 * rng.standard_normal((nx, nz))
    rho = 310.0 * vp ** 0.25
    return vp.astype(np.float32), rho.astype(np.float32)


# 300 rows + 2 x 24 sponge: strips of 112 rows, some clear of the z-sponge
# (literal-coefficient path) and some not; receivers on the first and last
# rows and columns reach the rows where the operator falls back to the
# reference's 4th-order and edge rows.
NX, NZ, NB, D = 130, 300, 24, 10.0
T, DT, DDT, F = 0.3, 0.001, 0.002, 18.0


def _shots(m):
    from seis2d_b200 import Shot
    rec = np.concatenate([np.stack([np.arange(NX) * D, np.full(NX, 0.0)], 1),
                          np.stack([np.arange(NX) * D, np.full(NX, (NZ - 1) * D)], 1),
                          np.stack([np.full(NZ, (NX - 1) * D), np.arange(NZ) * D], 1)]).astype(np.float32)
    return [Shot(m, src, rec) for src in ((650.0, 20.0), (30.0, 1500.0), (1100.0, 2900.0))], rec


def _wave():
    from seis2d_b200 import Wave
    return Wave(T, DT, DDT, F)


def _oracle(vp, rho, src, rec, precision):
    p = O.Params(NX, NZ, NB, D, D, T, DT, DDT, F, 0, 8)
    return O.forward(p, vp, rho, src, rec[:, 0], rec[:, 1], precision)


def test_forward_matches_oracle(ctx):
    vp, rho = _model(NX, NZ, 1)
    m = ctx.model(vp, rho, D, D, NB, fd_order=8)
    shots, rec = _shots(m)
    got = ctx.forward(shots, _wave())
    st = ctx.last_stats
    assert st.variant in (7, 8, 9)
    for s, g in zip(shots, got):
        assert O.rel_l2(g, _oracle(vp, rho, s.src, rec, O.F64)) <= TOL
        assert O.rel_l2(g, _oracle(vp, rho, s.src, rec, O.F32)) <= 2e-6
    # not the 4th-order traces
    m4 = ctx.model(vp, rho, D, D, NB)
    four = ctx.forward(_shots(m4)[0], _wave())
    assert O.rel_l2(got[0], four[0]) > 1e-3
    m.release()
    m4.release()


def test_tuned_fixed_plain_and_stepwise_runs_agree():
    """The three launch forms the autotuner chooses between (register windows
    at 3 and 2 blocks per SM, shared-memory windows at 4), shot after shot,
    and launches without a graph compute the same bits."""
    from seis2d_b200 import Context
    c = Context(0)
    forced = {}
    try:
        vp, rho = _model(NX, NZ, 2)
        m = c.model(vp, rho, D, D, NB, fd_order=8)
        shots, _ = _shots(m)
        tuned = c.forward(shots, _wave())
        s1 = c.last_stats
        plain = c.forward(shots, _wave(), plain=True)
        nograph = c.forward(shots, _wave(), graph=False)
        c.set_option("autotune", 0)
        fixed = c.forward(shots, _wave())
        s2 = c.last_stats
        for v in (7, 8, 9):
            c.set_option("variant", v)
            forced[v] = (c.forward(shots, _wave()), c.last_stats.variant)
    finally:
        c.close()
    assert s1.autotuned == 1 and s1.variant in (7, 8, 9) and s2.variant == 7
    for a, b, d, f in zip(tuned, plain, nograph, fixed):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, d)
        np.testing.assert_array_equal(a, f)
    for v, (traces, used) in forced.items():
        assert used == v
        for a, f in zip(tuned, traces):
            np.testing.assert_array_equal(a, f)


def test_uneven_models_and_continuation(ctx):
    """Two order-8 models of different sizes in one launch sequence, run in
    two continuation calls recording into one device buffer."""
    import torch
    from seis2d_b200 import Shot, derive_steps
    va, ra = _model(90, 60, 3)
    vb, rb = _model(150, 110, 4)
    ma = ctx.model(va, ra, D, D, 30, fd_order=8)
    mb = ctx.model(vb, rb, D, D, 30, fd_order=8)
    reca = np.stack([np.arange(90) * D, np.full(90, 20.0)], 1).astype(np.float32)
    recb = np.stack([np.arange(150) * D, np.full(150, 20.0)], 1).astype(np.float32)
    shots = [Shot(ma, (400.0, 30.0), reca), Shot(mb, (700.0, 30.0), recb), Shot(mb, (200.0, 500.0), recb)]
    nt = derive_steps(_wave())["real_nt"]
    out = torch.zeros((90 + 150 + 150) * nt, dtype=torch.float32, device="cuda")
    ctx.forward(shots, _wave(), kt_begin=0, kt_count=123, out=out)
    ctx.forward(shots, _wave(), kt_begin=123, kt_count=0, out=out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    whole = ctx.forward(shots, _wave())
    np.testing.assert_array_equal(got[:90 * nt].reshape(90, nt), whole[0])
    for s, g in zip(shots, whole):
        nx, nz = s.model.nx, s.model.nz
        v, r = (va, ra) if nx == 90 else (vb, rb)
        p = O.Params(nx, nz, 30, D, D, T, DT, DDT, F, 0, 8)
        ref = O.forward(p, v, r, s.src, s.rec[:, 0], s.rec[:, 1], O.F64)
        assert O.rel_l2(g, ref) <= TOL
    ma.release()
    mb.release()


def test_mixed_orders_are_refused(ctx):
    from seis2d_b200 import Shot
    from seis2d_b200._lib import Seis2dError
    vp, rho = _model(60, 40, 5)
    m8 = ctx.model(vp, rho, D, D, 20, fd_order=8)
    m4 = ctx.model(vp, rho, D, D, 20)
    rec = np.stack([np.arange(60) * D, np.full(60, 20.0)], 1).astype(np.float32)
    with pytest.raises(Seis2dError):
        ctx.forward([Shot(m8, (300.0, 20.0), rec), Shot(m4, (300.0, 20.0), rec)], _wave())
    # the context still works after the refusal
    a = ctx.forward([Shot(m8, (300.0, 20.0), rec)], _wave())[0]
    p = O.Params(60, 40, 20, D, D, T, DT, DDT, F, 0, 8)
    assert O.rel_l2(a, O.forward(p, vp, rho, (300.0, 20.0), rec[:, 0], rec[:, 1], O.F64)) <= TOL
    m8.release()
    m4.release()


# gradient case (the 4th-order gradient tests' sizes)
GNX, GNZ, GNB = 60, 40, 32
GRAD_TOL = 1e-4   # rel-L2 of the FP32 gradient against the FP64 adjoint


def _gwave():
    from seis2d_b200 import Wave
    return Wave(0.3, 0.001, 0.002, 20.0)


def _ggeom(sx=300.0):
    rx = np.arange(2, GNX - 2, 2) * D
    return (sx, 20.0), np.stack([rx, np.full(rx.size, 20.0)], 1).astype(np.float32)


def test_order8_gradient_matches_fp64_adjoint(ctx):
    from seis2d_b200 import Shot
    vp, rho = _model(GNX, GNZ, 7)
    src, rec = _ggeom()
    p = O.Params(GNX, GNZ, GNB, D, D, 0.3, 0.001, 0.002, 20.0, 0, 8)
    nt = O.derive(p)["real_nt"]
    adj = np.random.default_rng(7).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, GNB, fd_order=8)
    g = ctx.gradient([Shot(m, src, rec)], _gwave(), adj)
    ref = O.gradient(p, vp, rho, src, rec[:, 0], rec[:, 1], adj.astype(np.float64))
    e_vp = O.rel_l2(g.grad_vp, ref["grad_vp"])
    e_rho = O.rel_l2(g.grad_rho, ref["grad_rho"])
    assert e_vp <= GRAD_TOL and e_rho <= GRAD_TOL, (e_vp, e_rho)
    k = O.derive(p)
    ix, iz = int(src[0] * np.float32(1 / D)), int(src[1] * np.float32(1 / D))
    ks = float(vp[ix, iz]) ** 2 * float(rho[ix, iz])
    gw_ref = ref["src_adj"] * (float(np.float32(0.001)) * ks / float(np.float32(D * D)))
    n = min(k["nts"] + 1, k["fd_nt"])
    assert O.rel_l2(g.grad_wavelet[0, :n], gw_ref[:n]) <= GRAD_TOL
    m.release()


def test_order8_gradient_segments_and_dot_product(ctx):
    """Checkpoint segments change no bit; <F w, r> = <w, F^T r> for the map
    from source samples to traces (FP64 inner products)."""
    from seis2d_b200 import Shot
    vp, rho = _model(GNX, GNZ, 9)
    src, rec = _ggeom(350.0)
    nt = O.derive(O.Params(GNX, GNZ, GNB, D, D, 0.3, 0.001, 0.002, 20.0))["real_nt"]
    rng = np.random.default_rng(21)
    r = rng.standard_normal((rec.shape[0], nt)).astype(np.float32)
    w = rng.standard_normal(180)
    m = ctx.model(vp, rho, D, D, GNB, fd_order=8)
    whole = ctx.gradient([Shot(m, src, rec)], _gwave(), r, wavelet=w)
    try:
        ctx.set_option("grad_segment", 37)
        seg = ctx.gradient([Shot(m, src, rec)], _gwave(), r, wavelet=w)
    finally:
        ctx.set_option("grad_segment", 0)
    assert seg.stats.grad_segment == 37
    np.testing.assert_array_equal(seg.grad_vp, whole.grad_vp)
    np.testing.assert_array_equal(seg.grad_rho, whole.grad_rho)
    d = ctx.forward([Shot(m, src, rec)], _gwave(), wavelet=w)[0]
    lhs = float(np.sum(d.astype(np.float64) * r.astype(np.float64)))
    rhs = float(np.sum(w * whole.grad_wavelet[0, :w.size]))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)
    m.release()


def test_jobcard_order8(tmp_path, monkeypatch):
    from cases import model
    from seis2d_b200 import driver as Dv
    from seis2d_b200 import formats as Fm
    monkeypatch.chdir(tmp_path)
    z = np.load(os.path.join(GOLDEN, "twolayer_split_nb32.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    Fm.write_model("vp.bin", vp)
    Fm.write_model("rho.bin", rho)
    card = str(z["jobcard"])
    assert '"Order of FD Operator" : "4"' in card
    (tmp_path / "case.json").write_text(card.replace('"Order of FD Operator" : "4"', '"Order of FD Operator" : "8"'))
    (tmp_path / "geom.txt").write_text(str(z["geomfile"]))
    os.makedirs("out", exist_ok=True)
    Dv.run_jobcard("case.json", nb=c["nb"], naming="cpu")
    got = Fm.read_seismogram("out/case_seismogram.bin", z["rec"].shape[0])
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"], 0, 8)
    ref = O.forward(p, vp, rho, z["src"], z["rec"][:, 0], z["rec"][:, 1], O.F64)
    assert O.rel_l2(got, ref) <= TOL
    assert O.rel_l2(got, z["seis"]) > 1e-3


def test_order8_streaming_adjoint_on_interior_strips(ctx):
    """A grid tall and wide enough for strips and segments clear of the sponge,
    so the streaming 8th-order adjoint (the default) takes its literal-
    coefficient paths as well as the general ones: its gradient is within the
    bar of the FP64 8th-order adjoint, and agrees with the two cell-parallel
    passes to rounding (the same sums per cell; the compiler may fuse a product
    and a sum differently in the two)."""
    from seis2d_b200 import Shot, Wave
    nx, nz, nb = 160, 400, 32
    vp, rho = _model(nx, nz, 13)
    wave = Wave(0.12, 0.001, 0.002, 20.0)
    src = (800.0, 20.0)
    rx = np.arange(4, nx - 4, 3) * D
    rec = np.stack([rx, np.full(rx.size, 20.0)], 1).astype(np.float32)
    p = O.Params(nx, nz, nb, D, D, 0.12, 0.001, 0.002, 20.0, 0, 8)
    nt = O.derive(p)["real_nt"]
    adj = np.random.default_rng(29).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, nb, fd_order=8)
    out = {}
    try:
        for form in (0, 1):
            ctx.set_option("adjoint8_form", form)
            out[form] = ctx.gradient([Shot(m, src, rec)], wave, adj)
    finally:
        ctx.set_option("adjoint8_form", 0)
    ref = O.gradient(p, vp, rho, src, rec[:, 0], rec[:, 1], adj.astype(np.float64))
    assert O.rel_l2(out[0].grad_vp, ref["grad_vp"]) <= GRAD_TOL
    assert O.rel_l2(out[0].grad_rho, ref["grad_rho"]) <= GRAD_TOL
    assert O.rel_l2(out[0].grad_vp, out[1].grad_vp) <= 1e-6
    assert O.rel_l2(out[0].grad_rho, out[1].grad_rho) <= 1e-6
    m.release()
