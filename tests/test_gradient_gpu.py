"""FWI gradient (s2d_gradient, hand-written adjoint) against:
  * the FP64 CPU discrete adjoint of the reference scheme (oracle/s2d_oracle.c,
    itself checked by its own dot-product and finite-difference tests),
  * the dot-product test of the wave propagation (source samples -> traces),
  * central finite differences of the FP64 forward on 16 random cells,
  * itself with forced checkpoint segments (recompute must not change a bit),
  * torch autograd through seis2d_b200.autograd.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NX, NZ, NB, D = 60, 40, 32, 10.0
T, DT, DDT, F = 0.3, 0.001, 0.002, 20.0
GRAD_TOL = 1e-4   # rel-L2 of the FP32 gradient field against the FP64 adjoint


def _model(seed=3):
    rng = np.random.default_rng(seed)
    x = np.linspace(0, 1, NX)[:, None]
    z = np.linspace(0, 1, NZ)[None, :]
    vp = 1800 + 900 * z + 80 * np.sin(6 * x) * np.cos(5 * z) + 20 * rng.standard_normal((NX, NZ))
    rho = 1300 + 600 * z + 40 * np.cos(4 * x + 3 * z)
    return vp.astype(np.float32), rho.astype(np.float32)


def _geom(sx=300.0):
    rx = np.arange(2, NX - 2, 2) * D
    rec = np.stack([rx, np.full(rx.size, 20.0)], 1).astype(np.float32)
    return (sx, 20.0), rec


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _wave():
    from seis2d_b200 import Wave
    return Wave(T, DT, DDT, F)


def test_gradient_matches_fp64_adjoint(ctx):
    from seis2d_b200 import Shot
    vp, rho = _model()
    src, rec = _geom()
    p = O.Params(NX, NZ, NB, D, D, T, DT, DDT, F)
    nt = O.derive(p)["real_nt"]
    adj = np.random.default_rng(7).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB)
    g = ctx.gradient([Shot(m, src, rec)], _wave(), adj)
    ref = O.gradient(p, vp, rho, src, rec[:, 0], rec[:, 1], adj.astype(np.float64))
    e_vp = O.rel_l2(g.grad_vp, ref["grad_vp"])
    e_rho = O.rel_l2(g.grad_rho, ref["grad_rho"])
    assert e_vp <= GRAD_TOL and e_rho <= GRAD_TOL, (e_vp, e_rho)
    # source-wavelet gradient: the FP64 transpose of the injection
    k = O.derive(p)
    ix, iz = int(src[0] * np.float32(1 / D)), int(src[1] * np.float32(1 / D))
    ks = float(vp[ix, iz]) ** 2 * float(rho[ix, iz])
    gw_ref = ref["src_adj"] * (float(np.float32(DT)) * ks / float(np.float32(D * D)))
    n = min(k["nts"] + 1, k["fd_nt"])
    assert O.rel_l2(g.grad_wavelet[0, :n], gw_ref[:n]) <= GRAD_TOL


def test_checkpoint_segments_do_not_change_the_gradient(ctx):
    from seis2d_b200 import Shot
    vp, rho = _model(5)
    src, rec = _geom(350.0)
    nt = O.derive(O.Params(NX, NZ, NB, D, D, T, DT, DDT, F))["real_nt"]
    adj = np.random.default_rng(11).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB)
    whole = ctx.gradient([Shot(m, src, rec)], _wave(), adj)
    assert whole.stats.grad_segment == 300
    try:
        ctx.set_option("grad_segment", 37)
        seg = ctx.gradient([Shot(m, src, rec)], _wave(), adj)
    finally:
        ctx.set_option("grad_segment", 0)
    assert seg.stats.grad_segment == 37
    np.testing.assert_array_equal(seg.grad_vp, whole.grad_vp)
    np.testing.assert_array_equal(seg.grad_rho, whole.grad_rho)


def test_dot_product_source_to_traces(ctx):
    """<F w, r> = <w, F^T r> for the linear map from source samples w to the
    recorded traces, F^T r being the adjoint's dJ/dw; FP64 inner products."""
    from seis2d_b200 import Shot
    vp, rho = _model(9)
    src, rec = _geom(250.0)
    steps = O.derive(O.Params(NX, NZ, NB, D, D, T, DT, DDT, F))
    rng = np.random.default_rng(21)
    w = rng.standard_normal(180)
    r = rng.standard_normal((rec.shape[0], steps["real_nt"])).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB)
    d = ctx.forward([Shot(m, src, rec)], _wave(), wavelet=w)[0]
    g = ctx.gradient([Shot(m, src, rec)], _wave(), r, wavelet=w)
    lhs = float(np.sum(d.astype(np.float64) * r.astype(np.float64)))
    rhs = float(np.sum(w * g.grad_wavelet[0, :w.size]))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)


def test_gradient_central_differences_16_cells(ctx):
    """dJ/dvp, dJ/drho at 16 random cells against central differences of the
    FP64 misfit J = 0.5 ||d(m) - d_obs||^2 (the oracle's forward)."""
    from seis2d_b200 import Shot
    vp, rho = _model(13)
    src, rec = _geom(300.0)
    p = O.Params(NX, NZ, NB, D, D, T, DT, DDT, F)
    vp_true = vp.copy()
    vp_true[25:35, 15:25] += 60.0
    dobs = O.gradient(p, vp_true, rho, src, rec[:, 0], rec[:, 1], None)["seis64"]

    def J(v, r):
        s = O.gradient(p, v, r, src, rec[:, 0], rec[:, 1], None)["seis64"]
        return 0.5 * np.sum((s - dobs) ** 2)

    m = ctx.model(vp, rho, D, D, NB)
    g = ctx.gradient([Shot(m, src, rec)], _wave(), dobs.astype(np.float32), misfit=True)
    rng = np.random.default_rng(5)
    cells = [(int(i), int(j)) for i, j in zip(rng.integers(10, NX - 10, 16), rng.integers(3, NZ - 5, 16))]
    for name, arr, grad in (("vp", vp, g.grad_vp), ("rho", rho, g.grad_rho)):
        scale = np.abs(grad).max()
        for i, j in cells:
            eps = float(arr[i, j]) * 2e-3
            a1, a2 = arr.copy(), arr.copy()
            a1[i, j] += eps
            a2[i, j] -= eps
            jp = J(a1, rho) if name == "vp" else J(vp, a1)
            jm = J(a2, rho) if name == "vp" else J(vp, a2)
            fd = (jp - jm) / (float(a1[i, j]) - float(a2[i, j]))
            assert abs(fd - grad[i, j]) <= 2e-3 * scale + 1e-3 * abs(fd), (name, i, j, fd, grad[i, j], scale)


def test_misfit_mode_equals_residual_as_adjoint_source(ctx):
    from seis2d_b200 import Shot
    vp, rho = _model(17)
    src, rec = _geom(320.0)
    m = ctx.model(vp, rho, D, D, NB)
    shot = [Shot(m, src, rec)]
    d = ctx.forward(shot, _wave())[0]
    dobs = (0.8 * d + 1.0).astype(np.float32)
    a = ctx.gradient(shot, _wave(), dobs, misfit=True, want_seis=True)
    b = ctx.gradient(shot, _wave(), (d - dobs).astype(np.float32))
    np.testing.assert_array_equal(a.seis.reshape(d.shape), d)
    assert abs(a.misfit - 0.5 * np.sum((d.astype(np.float64) - dobs) ** 2)) <= 1e-6 * a.misfit
    np.testing.assert_array_equal(a.grad_vp, b.grad_vp)
    np.testing.assert_array_equal(a.grad_rho, b.grad_rho)


def test_gradient_sums_over_shots(ctx):
    from seis2d_b200 import Shot
    vp, rho = _model(19)
    m = ctx.model(vp, rho, D, D, NB)
    nt = O.derive(O.Params(NX, NZ, NB, D, D, T, DT, DDT, F))["real_nt"]
    rng = np.random.default_rng(23)
    shots, adjs = [], []
    for sx in (150.0, 300.0, 450.0):
        src, rec = _geom(sx)
        shots.append(Shot(m, src, rec))
        adjs.append(rng.standard_normal((rec.shape[0], nt)).astype(np.float32))
    both = ctx.gradient(shots, _wave(), np.concatenate([a.ravel() for a in adjs]))
    singles = [ctx.gradient([s], _wave(), a) for s, a in zip(shots, adjs)]
    total_vp = sum(s.grad_vp.astype(np.float64) for s in singles)
    total_rho = sum(s.grad_rho.astype(np.float64) for s in singles)
    assert O.rel_l2(both.grad_vp, total_vp) <= 1e-6
    assert O.rel_l2(both.grad_rho, total_rho) <= 1e-6


def test_torch_autograd(ctx):
    import torch
    from seis2d_b200 import Wave
    from seis2d_b200.autograd import modelled_seismograms
    vp, rho = _model(29)
    src, rec = _geom(300.0)
    geometry = [(src, rec)]
    wave = _wave()
    vp_t = torch.from_numpy(vp).cuda().requires_grad_(True)
    rho_t = torch.from_numpy(rho).cuda().requires_grad_(True)
    seis = modelled_seismograms(vp_t, rho_t, geometry, wave, D, D, NB)
    dobs = torch.zeros_like(seis) + 0.5
    loss = 0.5 * ((seis - dobs) ** 2).sum()
    loss.backward()
    from seis2d_b200 import Shot
    m = ctx.model(vp, rho, D, D, NB)
    g = ctx.gradient([Shot(m, src, rec)], wave, dobs.detach().cpu().numpy(), misfit=True)
    assert O.rel_l2(vp_t.grad.cpu().numpy(), g.grad_vp) <= 1e-6
    assert O.rel_l2(rho_t.grad.cpu().numpy(), g.grad_rho) <= 1e-6


def test_gradient_allreduce_through_nccl(ctx):
    """seis2d_b200.sharding.gradient_allreduce on a one-rank NCCL group: the
    device images and the misfit go through the all-reduce unchanged (to the
    rounding of the shots' atomic accumulation)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    from seis2d_b200 import Shot
    from seis2d_b200.sharding import gradient_allreduce
    vp, rho = _model(31)
    m = ctx.model(vp, rho, D, D, NB)
    shots = [Shot(m, *_geom(sx)) for sx in (200.0, 330.0, 460.0)]
    d = torch.cat([torch.from_numpy(ctx.forward([s], _wave())[0].ravel()) for s in shots]).cuda() * 0.7
    ref = ctx.gradient(shots, _wave(), d, misfit=True)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        gv, gr, mis = gradient_allreduce(ctx, shots, _wave(), d)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    # the shots' imaging terms meet in one accumulator pair through atomics
    # whose order is not fixed: two runs agree to rounding
    assert O.rel_l2(gv.cpu().numpy(), ref.grad_vp) <= 1e-6
    assert O.rel_l2(gr.cpu().numpy(), ref.grad_rho) <= 1e-6
    assert abs(mis - ref.misfit) <= 1e-9 * ref.misfit


def test_products_variants_give_the_same_gradient(ctx):
    """The product-writing recompute with plain loads (3) and with the next
    column prefetched (19, the default) share the update arithmetic: one
    shot's gradient is the same bit for bit."""
    from seis2d_b200 import Shot
    vp, rho = _model(41)
    src, rec = _geom(310.0)
    nt = O.derive(O.Params(NX, NZ, NB, D, D, T, DT, DDT, F))["real_nt"]
    adj = np.random.default_rng(43).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB)
    try:
        ctx.set_option("grad_segment", 37)
        out = {}
        for pv in (3, 19):
            ctx.set_option("products_variant", pv)
            out[pv] = ctx.gradient([Shot(m, src, rec)], _wave(), adj)
    finally:
        ctx.set_option("products_variant", 19)
        ctx.set_option("grad_segment", 0)
    np.testing.assert_array_equal(out[3].grad_vp, out[19].grad_vp)
    np.testing.assert_array_equal(out[3].grad_rho, out[19].grad_rho)


def test_adjoint_forms_give_the_same_gradient(ctx):
    """The adjoint kernel's builds (3 blocks per SM; 2; 2 with the next
    column prefetched; 3 and 2 with the column inputs copied into shared
    memory ahead, the first the default) share its arithmetic: one shot's
    gradient is the same bit for bit."""
    from seis2d_b200 import Shot
    vp, rho = _model(47)
    src, rec = _geom(290.0)
    nt = O.derive(O.Params(NX, NZ, NB, D, D, T, DT, DDT, F))["real_nt"]
    adj = np.random.default_rng(53).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, D, D, NB)
    out = {}
    try:
        for ab in (3, 2, 12, 13, 14, 15):
            ctx.set_option("adjoint_blocks", ab)
            out[ab] = ctx.gradient([Shot(m, src, rec)], _wave(), adj)
    finally:
        ctx.set_option("adjoint_blocks", 13)
    for ab in (2, 12, 13, 14, 15):
        np.testing.assert_array_equal(out[ab].grad_vp, out[3].grad_vp)
        np.testing.assert_array_equal(out[ab].grad_rho, out[3].grad_rho)
