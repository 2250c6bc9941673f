"""s2d_forward_static: forward modelling for callers that cannot allocate
device memory (services that reserve their memory at start-up, programs whose
own allocator holds the device memory, loops that cannot afford cudaMalloc's
synchronisation).  It works in a fixed static device array instead.

Checked through the C ABI against the allocating entry point s2d_forward on the
same inputs, on two calls in a row (the array keeps the last call's contents,
so the second call shows that everything that must start at zero is cleared).
This file is collected last so that a failure here leaves every other test
already run.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from cases import model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the seismogram tolerance of the forward tests
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _case(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    return z, c, vp, rho


def _static_call(c, vp, rho, src, rec, out, flags=0, vp_ptr=None, rho_ptr=None, out_ptr=None):
    from seis2d_b200 import _lib as L
    recs = np.ascontiguousarray(rec, np.float32)
    shot = L.Shot(0, L.Coord(float(src[0]), float(src[1])), recs.shape[0], recs.ctypes.data_as(C.POINTER(L.Coord)))
    wave = L.Wave(c["T"], c["dt"], c["ddt"], c["f"])
    err = C.create_string_buffer(512)
    rc = L.lib().s2d_forward_static(
        0, c["nx"], c["nz"], c["dx"], c["dz"], c["nb"],
        vp_ptr if vp_ptr is not None else C.c_void_p(vp.ctypes.data),
        rho_ptr if rho_ptr is not None else C.c_void_p(rho.ctypes.data),
        C.byref(wave), C.byref(shot),
        out_ptr if out_ptr is not None else C.c_void_p(out.ctypes.data),
        flags, None, err, 512)
    return rc, err.value.decode()


@pytest.mark.parametrize("name", ["twolayer_split_nb32", "gradient_endonleft_nb40"])
def test_static_entry_matches_allocating_entry_twice(name):
    from seis2d_b200 import Context, Shot, Wave
    z, c, vp, rho = _case(name)
    with Context(0) as ctx:
        m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
        ref = ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], Wave(c["T"], c["dt"], c["ddt"], c["f"]))[0]
    for call in range(2):
        out = np.full(ref.size, np.nan, np.float32)
        rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], out)
        assert rc == 0, msg
        got = out.reshape(ref.shape)
        assert O.rel_l2(got, ref) <= TOL, (call, O.rel_l2(got, ref))
        assert O.rel_l2(got, z["seis"]) <= TOL


def test_static_entry_device_buffers():
    import torch
    from seis2d_b200 import _lib as L
    z, c, vp, rho = _case("edges_explicit_nb32")
    host = np.zeros(z["seis"].size, np.float32)
    rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], host)
    assert rc == 0, msg
    vp_d, rho_d = torch.from_numpy(vp).cuda(), torch.from_numpy(rho).cuda()
    out_d = torch.full((host.size,), float("nan"), dtype=torch.float32, device="cuda")
    rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], None, flags=L.S2D_MODEL_DEVICE | L.S2D_SEIS_DEVICE,
                           vp_ptr=C.c_void_p(vp_d.data_ptr()), rho_ptr=C.c_void_p(rho_d.data_ptr()),
                           out_ptr=C.c_void_p(out_d.data_ptr()))
    assert rc == 0, msg
    assert O.rel_l2(out_d.cpu().numpy(), host) <= TOL


def test_static_entry_rejects_oversized_jobs():
    from seis2d_b200 import _lib as L
    z, c, vp, rho = _case("twolayer_split_nb32")
    big = dict(c, nx=3000, nz=3000)
    vpb = np.full((3000, 3000), 2000.0, np.float32)
    out = np.zeros(1, np.float32)
    rc, msg = _static_call(big, vpb, vpb, (100.0, 10.0), np.array([[10.0, 10.0]], np.float32), out)
    assert rc == L.S2D_ERR_NOMEM
    assert "needs" in msg and "static scratch holds" in msg
