"""Parity of the CUDA forward path (through the C ABI) with the reference.

Golden seismograms were produced by the reference CPU binary itself
(tests/golden/make_golden.py); the oracle (oracle/s2d_oracle.c, bit-exact
with the reference on those cases) covers the other inputs.  Bar: relative
L2 of the FP32 seismogram against the reference's FP64 one <= 1e-5.
"""
import json
import os

import numpy as np
import pytest

from cases import CASES, model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # seismogram rel-L2, FP32 CUDA vs FP64 reference
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def ctx():
    from seis2d_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    return z, c, vp, rho


def _wave(c):
    from seis2d_b200 import Wave
    return Wave(c["T"], c["dt"], c["ddt"], c["f"])


VARIANTS = {"bulk": 0, "ldg": 1, "bulk128": 2, "ldg128": 4, "twostep": 5, "tma": 11, "async": 12, "ldgu4": 14, "ldgpf": 15, "ldgpf4": 16, "ldgpfu4": 17, "ldgpfu3": 18, "persist": 20}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_parity(ctx, name, variant):
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden(name)
    ctx.set_option("variant", VARIANTS[variant])
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    try:
        seis = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], _wave(c))[0]
    finally:
        ctx.set_option("autotune", 1)
    ref = z["seis"]
    assert seis.shape == ref.shape
    err = O.rel_l2(seis, ref)
    assert err <= TOL, err
    # against the FP32 CPU restatement of the same arithmetic: tighter
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"])
    s32 = O.forward(p, vp, rho, z["src"], z["rec"][:, 0], z["rec"][:, 1], O.F32)
    assert O.rel_l2(seis, s32) <= 2e-6
    m.release()


def test_state_after_few_steps_matches_oracle(ctx):
    """Cell-by-cell p after 1, 2 and 10 steps on an odd-sized grid, through
    the seismogram of a receiver at every cell of a few rows and columns."""
    from seis2d_b200 import Shot, Wave
    nx, nz, nb = 37, 29, 32
    vp = np.full((nx, nz), 2000.0, np.float32)
    vp[:, 15:] = 2600.0
    rho = np.full((nx, nz), 1500.0, np.float32)
    rho[20:, :] = 2100.0
    dx = dz = 10.0
    m = ctx.model(vp, rho, dx, dz, nb)
    # receivers on every physical cell
    xs, zs = np.meshgrid(np.arange(nx) * dx, np.arange(nz) * dz, indexing="ij")
    rec = np.stack([xs.ravel(), zs.ravel()], 1).astype(np.float32)
    wave = Wave(0.012, 0.001, 0.001, 25.0)
    seis = ctx.forward([Shot(m, (180.0, 60.0), rec)], wave)[0]  # [ncell][12]
    p = O.Params(nx, nz, nb, dx, dz, 0.012, 0.001, 0.001, 25.0)
    ref = O.forward(p, vp, rho, (180.0, 60.0), rec[:, 0], rec[:, 1], O.F64)
    for k in (0, 1, 9):
        a, b = seis[:, k], ref[:, k]
        assert O.rel_l2(a, b) < 1e-5, (k, O.rel_l2(a, b))


def test_plain_batched_graph_modes_agree(ctx):
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("twolayer_split_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    shots = [Shot(m, (x, 20.0), z["rec"]) for x in (300.0, 800.0, 1200.0)]
    w = _wave(c)
    batched = ctx.forward(shots, w)
    plain = ctx.forward(shots, w, plain=True)
    nograph = ctx.forward(shots, w, graph=False)
    for a, b, d in zip(batched, plain, nograph):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, d)
    # the middle shot is the golden one
    assert O.rel_l2(batched[1], z["seis"]) <= TOL


def test_continuation_equals_single_call(ctx):
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("gradient_endonleft_nb40")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    w = _wave(c)
    shots = [Shot(m, tuple(z["src"]), z["rec"])]
    whole = ctx.forward(shots, w)[0]
    nrec, nt = whole.shape
    out = np.full(nrec * nt, np.nan, np.float32)
    k = 0
    for n in (1, 97, 200, 0):  # 0: to the end
        ctx.forward(shots, w, kt_begin=k, kt_count=n, out=out)
        k += n
    np.testing.assert_array_equal(out.reshape(nrec, nt), whole)


def test_uneven_models_in_one_batch(ctx):
    """Shots on models of different sizes in one launch sequence equal the
    same shots run alone."""
    from seis2d_b200 import Shot
    shots, singles = [], []
    w = None
    for name in ("twolayer_split_nb32", "layers_endonright_near_nb32", "corner_source_nb40"):
        z, c, vp, rho = _golden(name)
        w = _wave(c) if w is None else w
        m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
        shots.append(Shot(m, tuple(z["src"]), z["rec"]))
    both = ctx.forward(shots, w)
    for s, got in zip(shots, both):
        alone = ctx.forward([s], w)[0]
        np.testing.assert_array_equal(got, alone)


def test_device_output_matches_host(ctx):
    import torch
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("edges_explicit_nb32")
    m = ctx.model(torch.from_numpy(vp).cuda(), torch.from_numpy(rho).cuda(), c["dx"], c["dz"], c["nb"])
    w = _wave(c)
    host = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], w)[0]
    dev = torch.zeros(host.size, dtype=torch.float32, device="cuda")
    ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], w, out=dev)
    np.testing.assert_array_equal(dev.cpu().numpy().reshape(host.shape), host)
    assert O.rel_l2(host, z["seis"]) <= TOL


def test_custom_wavelet_equals_ricker(ctx):
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("twolayer_split_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"])
    w = O.ricker(p)  # nts samples; the reference's sample at kt == nts is 0
    w = np.concatenate([w, [0.0]])
    a = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], _wave(c), wavelet=w)[0]
    b = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], _wave(c))[0]
    np.testing.assert_array_equal(a, b)


def test_errors_are_statuses(ctx):
    from seis2d_b200 import Shot
    from seis2d_b200._lib import Seis2dError, S2D_ERR_GEOM, S2D_ERR_STATE
    z, c, vp, rho = _golden("twolayer_split_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    far = np.array([[1e6, 0.0]], np.float32)
    with pytest.raises(Seis2dError) as e:
        ctx.forward([Shot(m, (100.0, 0.0), far)], _wave(c))
    assert e.value.code == S2D_ERR_GEOM
    with pytest.raises(Seis2dError) as e:
        ctx.forward([Shot(m, (100.0, 0.0), z["rec"])], _wave(c), kt_begin=5, kt_count=5,
                    out=np.zeros(z["seis"].size, np.float32))
    assert e.value.code == S2D_ERR_STATE
    # context still usable after errors
    s = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], _wave(c))[0]
    assert O.rel_l2(s, z["seis"]) <= TOL


@pytest.mark.parametrize("stages,block,seg_len,order", [(2, 32, 16, 0), (3, 64, 24, 1), (8, 128, 0, 0),
                                                        (4, 96, 37, 1)])
def test_launch_shapes_agree(ctx, stages, block, seg_len, order):
    """Pipeline depth, block size and segment length change the schedule,
    never the numbers."""
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("layers_endonright_near_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    shot = [Shot(m, tuple(z["src"]), z["rec"])]
    base = ctx.forward(shot, _wave(c))[0]
    try:
        ctx.set_option("variant", 2)  # the bulk-copy pipeline: ring depth and block size matter
        ctx.set_option("stages", stages)
        ctx.set_option("block", block)
        ctx.set_option("seg_len", seg_len)
        ctx.set_option("task_order", order)
        got = ctx.forward(shot, _wave(c))[0]
    finally:
        ctx.set_option("stages", 3)
        ctx.set_option("block", 128)
        ctx.set_option("seg_len", 0)
        ctx.set_option("task_order", 1)
        ctx.set_option("autotune", 1)
    np.testing.assert_array_equal(got, base)


@pytest.mark.parametrize("seg_len", [4, 6])
@pytest.mark.parametrize("variant", [16, 15, 4, 5, 11, 12])
def test_short_segments_agree(ctx, variant, seg_len):
    """Segments of 4 and 6 columns (the layout picks them for small single
    grids: more tasks, fewer columns per task) give the same bits in every
    kernel family."""
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("layers_endonright_near_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    shot = [Shot(m, tuple(z["src"]), z["rec"])]
    base = ctx.forward(shot, _wave(c))[0]
    try:
        ctx.set_option("variant", variant)
        ctx.set_option("seg_len", seg_len)
        got = ctx.forward(shot, _wave(c))[0]
    finally:
        ctx.set_option("seg_len", 0)
        ctx.set_option("autotune", 1)
    np.testing.assert_array_equal(got, base)


@pytest.mark.parametrize("variant", [0, 11, 20])
def test_bounded_wait_reports_timeout_and_context_survives(ctx, variant):
    """A wait that never completes (the per-warp bulk-copy pipeline's stage,
    the TMA kernel's producer/consumer ring, the persistent kernel's grid
    barrier with one block not arriving): every wait is bounded, the kernel
    records the error and returns, the call reports S2D_ERR_TIMEOUT and the
    next call on the same context is correct."""
    from seis2d_b200 import Shot
    from seis2d_b200._lib import Seis2dError, S2D_ERR_TIMEOUT
    z, c, vp, rho = _golden("edges_explicit_nb32")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    shot = [Shot(m, tuple(z["src"]), z["rec"])]
    ctx.set_option("variant", variant)
    ctx.set_option("spin_limit", 256)
    ctx.set_option("inject_wait_fault", 1)
    try:
        with pytest.raises(Seis2dError) as e:
            ctx.forward(shot, _wave(c))
        assert e.value.code == S2D_ERR_TIMEOUT
    finally:
        ctx.set_option("inject_wait_fault", -1)
        ctx.set_option("spin_limit", 1 << 20)
        ctx.set_option("autotune", 1)
    good = ctx.forward(shot, _wave(c))[0]
    assert O.rel_l2(good, z["seis"]) <= TOL


def test_unknown_option_rejected(ctx):
    from seis2d_b200._lib import Seis2dError
    with pytest.raises(Seis2dError):
        ctx.set_option("no_such_knob", 1)
    with pytest.raises(Seis2dError):
        ctx.set_option("stages", 1)
    with pytest.raises(Seis2dError):
        ctx.set_option("block", 256)
    with pytest.raises(Seis2dError):
        ctx.set_option("autotune", 2)


def test_graph_chunking_is_transparent(ctx):
    """Replaying a short captured graph many times gives the same traces as
    step-by-step launches."""
    from seis2d_b200 import Shot
    z, c, vp, rho = _golden("gradient_endonleft_nb40")
    m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
    shot = [Shot(m, tuple(z["src"]), z["rec"])]
    plain = ctx.forward(shot, _wave(c), graph=False)[0]
    try:
        for chunk in (7, 1000):
            ctx.set_option("graph_chunk", chunk)
            np.testing.assert_array_equal(ctx.forward(shot, _wave(c))[0], plain)
    finally:
        ctx.set_option("graph_chunk", 64)


def _tall_grid(ctx, nshots=1):
    """A 70 x 420 model (nb 32) with vertical gradients and a step at row 250,
    receivers down a column and along the top; 450 steps."""
    from seis2d_b200 import Shot, Wave
    nx, nz, nb = 70, 420, 32
    z = np.arange(nz)[None, :] * 10.0
    vp = np.broadcast_to(1800.0 + 0.8 * z, (nx, nz)).astype(np.float32)
    vp[:, 250:] += 400.0
    rho = np.broadcast_to(1200.0 + 0.3 * z, (nx, nz)).astype(np.float32)
    rec = np.stack([np.full(40, 300.0), np.arange(40) * 100.0 + 50.0], 1)
    rec = np.concatenate([rec, np.stack([np.arange(0, 700, 20.0), np.full(35, 20.0)], 1)]).astype(np.float32)
    wave = Wave(0.45, 0.001, 0.002, 15.0)
    m = ctx.model(vp, rho, 10.0, 10.0, nb)
    shots = [Shot(m, (350.0 - 40.0 * k, 2000.0 + 30.0 * k), rec) for k in range(nshots)]
    p = O.Params(nx, nz, nb, 10.0, 10.0, 0.45, 0.001, 0.002, 15.0)
    return vp, rho, rec, wave, shots, p


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_tall_grid_fast_rows(ctx, variant):
    """A grid tall enough for strips clear of the z-sponge (the literal-row
    fast path): bit-identical with the fast path off, and within the bar of
    the FP64 oracle."""
    vp, rho, rec, wave, shot, p = _tall_grid(ctx)
    ctx.set_option("variant", VARIANTS[variant])
    try:
        fast = ctx.forward(shot, wave)[0]
        ctx.set_option("fast_rows", 0)
        slow = ctx.forward(shot, wave)[0]
    finally:
        ctx.set_option("fast_rows", 1)
        ctx.set_option("autotune", 1)
    np.testing.assert_array_equal(fast, slow)
    ref = O.forward(p, vp, rho, (350.0, 2000.0), rec[:, 0], rec[:, 1], O.F64)
    assert O.rel_l2(fast, ref) <= TOL


def test_variants_compute_the_same_bits(ctx):
    """Every step-kernel variant gives the same traces bit for bit (they share
    the update arithmetic), which is what lets the autotuner time candidates
    on the steps of a live run."""
    _, _, _, wave, shots, _ = _tall_grid(ctx, nshots=3)
    out = {}
    try:
        for name, v in sorted(VARIANTS.items()):
            ctx.set_option("variant", v)
            out[name] = np.concatenate(ctx.forward(shots, wave))
    finally:
        ctx.set_option("autotune", 1)
    for name in out:
        np.testing.assert_array_equal(out[name], out["ldg"], err_msg=name)


def test_autotuner_tunes_once_per_shape_and_keeps_the_bits():
    """A fresh context tunes on the first run of a batch shape (up to 56 of its
    steps, variant and task order), reuses the result for the next run of
    that shape, and the traces equal those of a fixed configuration."""
    from seis2d_b200 import Context
    c = Context(0)
    try:
        _, _, _, wave, shots, _ = _tall_grid(c, nshots=2)
        first = c.forward(shots, wave)
        s1 = c.last_stats
        again = c.forward(shots, wave)
        s2 = c.last_stats
        c.set_option("variant", 1)
        fixed = c.forward(shots, wave)
        s3 = c.last_stats
    finally:
        c.close()
    assert s1.autotuned == 1 and s2.autotuned == 0 and s3.autotuned == 0
    assert (s1.variant, s1.block, s1.stages, s1.task_order) == (s2.variant, s2.block, s2.stages, s2.task_order)
    assert s1.variant in (2, 4, 5, 11, 12, 15, 16) and s3.variant == 1
    assert s1.task_order in (0, 1) and (s1.task_order == 1 or s1.variant in (15, 16))
    for a, b, f in zip(first, again, fixed):
        np.testing.assert_array_equal(a, f)
        np.testing.assert_array_equal(b, f)


def test_autotuner_skips_short_calls():
    """A call with fewer steps than two rounds of trials runs untuned, and a
    later continuation with room tunes without changing the traces."""
    from seis2d_b200 import Context
    import torch
    from seis2d_b200 import derive_steps
    c = Context(0)
    try:
        _, _, rec, wave, shots, _ = _tall_grid(c, nshots=2)
        nt = derive_steps(wave)["real_nt"]
        out = torch.zeros(len(shots) * rec.shape[0] * nt, dtype=torch.float32, device="cuda")
        c.forward(shots, wave, kt_begin=0, kt_count=20, out=out)
        assert c.last_stats.autotuned == 0
        c.forward(shots, wave, kt_begin=20, kt_count=0, out=out)
        assert c.last_stats.autotuned == 1
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(len(shots), rec.shape[0], nt)
        c.set_option("variant", 1)
        ref = c.forward(shots, wave)
    finally:
        c.close()
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_odd_continuations_equal_one_run(ctx, variant):
    """A run cut into calls of 7 steps (odd: the two-step variant ends every
    call with a one-step launch and the next call starts from the other
    buffer) records the same traces as one call."""
    import torch
    from seis2d_b200 import derive_steps
    _, _, rec, wave, shots, _ = _tall_grid(ctx, nshots=2)
    steps = derive_steps(wave)
    nt, fd_nt = steps["real_nt"], steps["fd_nt"]
    ctx.set_option("variant", VARIANTS[variant])
    try:
        whole = np.concatenate(ctx.forward(shots, wave))
        out = torch.zeros(len(shots) * rec.shape[0] * nt, dtype=torch.float32, device="cuda")
        for k0 in range(0, fd_nt, 7):
            ctx.forward(shots, wave, kt_begin=k0, kt_count=7, out=out)
        torch.cuda.synchronize()
    finally:
        ctx.set_option("autotune", 1)
    np.testing.assert_array_equal(out.cpu().numpy().reshape(whole.shape), whole)
