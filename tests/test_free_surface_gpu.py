"""Free surface (S2D_MODEL_FREE_SURFACE, job card "Free surface" : "1") on
the GPU, against the CPU restatement with the same rule (kappa = 0 on padded
rows 0..nb; its physics is checked in tests/test_oracle_free_surface.py).

The reference parses the key and ignores it (src/src_cpu/json_parser.cpp:
236-244), so these cases have no reference output; the oracle is the bar, at
the same tolerances as the reference-parity tests.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5        # seismogram rel-L2, FP32 CUDA vs the FP64 oracle
GRAD_TOL = 1e-4   # gradient rel-L2, FP32 CUDA vs the FP64 adjoint
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _layered(nx, nz, seed):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[None, :]
    vp = np.where(z < nz // 3, 1800.0, np.where(z < 2 * nz // 3, 2400.0, 3000.0)) + 30 * rng.random((nx, nz))
    rho = 310.0 * vp ** 0.25
    return vp.astype(np.float32), rho.astype(np.float32)


VARIANTS = {"bulk": 0, "ldg": 1, "ldg128": 4, "twostep": 5}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_forward_matches_oracle(ctx, variant):
    """Three shots in one batch: a buried source, a source on the surface row
    (injects nothing: all-zero traces) and one in the sponge above it."""
    from seis2d_b200 import Shot, Wave
    nx, nz, nb, d = 150, 90, 40, 10.0
    T, dt, ddt, f = 0.35, 0.001, 0.002, 15.0
    vp, rho = _layered(nx, nz, 1)
    rx = np.arange(0, nx) * d
    rec = np.stack([rx, np.full(nx, 30.0)], 1).astype(np.float32)
    srcs = [(700.0, 40.0), (400.0, 0.0), (900.0, -50.0)]
    ctx.set_option("variant", VARIANTS[variant])
    try:
        m = ctx.model(vp, rho, d, d, nb, free_surface=True)
        got = ctx.forward([Shot(m, s, rec) for s in srcs], Wave(T, dt, ddt, f))
    finally:
        ctx.set_option("autotune", 1)
    p = O.Params(nx, nz, nb, d, d, T, dt, ddt, f, 1)
    ref = O.forward(p, vp, rho, srcs[0], rec[:, 0], rec[:, 1], O.F64)
    assert O.rel_l2(got[0], ref) <= TOL
    s32 = O.forward(p, vp, rho, srcs[0], rec[:, 0], rec[:, 1], O.F32)
    assert O.rel_l2(got[0], s32) <= 2e-6
    assert np.all(got[1] == 0) and np.all(got[2] == 0)
    # the surface changes the traces: the same shot without it differs
    p0 = O.Params(nx, nz, nb, d, d, T, dt, ddt, f, 0)
    assert O.rel_l2(got[0], O.forward(p0, vp, rho, srcs[0], rec[:, 0], rec[:, 1], O.F64)) > 0.05
    m.release()


def test_plain_and_batched_agree(ctx):
    from seis2d_b200 import Shot, Wave
    nx, nz, nb, d = 120, 70, 32, 10.0
    vp, rho = _layered(nx, nz, 2)
    rec = np.stack([np.arange(nx) * d, np.full(nx, 20.0)], 1).astype(np.float32)
    m = ctx.model(vp, rho, d, d, nb, free_surface=True)
    shots = [Shot(m, (x, 30.0), rec) for x in (200.0, 600.0, 1000.0)]
    w = Wave(0.3, 0.001, 0.001, 18.0)
    a = ctx.forward(shots, w)
    b = ctx.forward(shots, w, plain=True)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    m.release()


def test_gradient_matches_fp64_adjoint(ctx):
    from seis2d_b200 import Shot, Wave
    nx, nz, nb, d = 60, 40, 32, 10.0
    T, dt, ddt, f = 0.3, 0.001, 0.002, 20.0
    vp, rho = _layered(nx, nz, 3)
    rx = np.arange(2, nx - 2, 2) * d
    rec = np.stack([rx, np.full(rx.size, 20.0)], 1).astype(np.float32)
    src = (300.0, 30.0)
    p = O.Params(nx, nz, nb, d, d, T, dt, ddt, f, 1)
    nt = O.derive(p)["real_nt"]
    adj = np.random.default_rng(7).standard_normal((rec.shape[0], nt)).astype(np.float32)
    m = ctx.model(vp, rho, d, d, nb, free_surface=True)
    g = ctx.gradient([Shot(m, src, rec)], Wave(T, dt, ddt, f), adj)
    ref = O.gradient(p, vp, rho, src, rec[:, 0], rec[:, 1], adj.astype(np.float64))
    e_vp = O.rel_l2(g.grad_vp, ref["grad_vp"])
    e_rho = O.rel_l2(g.grad_rho, ref["grad_rho"])
    assert e_vp <= GRAD_TOL and e_rho <= GRAD_TOL, (e_vp, e_rho)
    # vp on the surface row only sets kappa that the surface holds at 0
    assert np.all(g.grad_vp[:, 0] == 0)
    m.release()


def test_jobcard_free_surface_flag(tmp_path, monkeypatch):
    """A card with "Free surface" : "1" runs with the surface; the same card
    with "0" still gives the reference's file."""
    from cases import model
    from seis2d_b200 import driver as D
    from seis2d_b200 import formats as F
    monkeypatch.chdir(tmp_path)
    z = np.load(os.path.join(GOLDEN, "twolayer_split_nb32.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    F.write_model("vp.bin", vp)
    F.write_model("rho.bin", rho)
    card = str(z["jobcard"])
    assert '"Free surface" : "0"' in card
    (tmp_path / "case.json").write_text(card.replace('"Free surface" : "0"', '"Free surface" : "1"'))
    (tmp_path / "geom.txt").write_text(str(z["geomfile"]))
    os.makedirs("out", exist_ok=True)
    D.run_jobcard("case.json", nb=c["nb"], naming="cpu")
    got = F.read_seismogram("out/case_seismogram.bin", z["rec"].shape[0])
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"], 1)
    ref = O.forward(p, vp, rho, z["src"], z["rec"][:, 0], z["rec"][:, 1], O.F64)
    assert O.rel_l2(got, ref) <= TOL
    assert O.rel_l2(got, z["seis"]) > 0.05
    (tmp_path / "case.json").write_text(card)
    D.run_jobcard("case.json", nb=c["nb"], naming="cpu")
    assert O.rel_l2(F.read_seismogram("out/case_seismogram.bin", z["rec"].shape[0]), z["seis"]) <= TOL
