"""s2d_forward_static: forward modelling for callers that cannot allocate
device memory (services that reserve their memory at start-up, programs whose
own allocator holds the device memory, loops that cannot afford cudaMalloc's
synchronisation).  It works in a fixed static device array instead.

Checked through the C ABI against the allocating entry point s2d_forward on the
same inputs, on two calls in a row (the array keeps the last call's contents,
so the second call shows that everything that must start at zero is cleared).
Both entries run the same plain-load arithmetic, so the traces must be equal
bit for bit.  Host and device pointers are accepted independently for the
model and for the seismogram.  This file is collected last so that a failure
here leaves every other test already run.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from cases import model
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the seismogram tolerance of the forward tests (against the reference)
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


def _allocating(z, c, vp, rho):
    from seis2d_b200 import Context, Shot, Wave
    with Context(0) as ctx:
        m = ctx.model(vp, rho, c["dx"], c["dz"], c["nb"])
        return ctx.forward([Shot(m, tuple(z["src"]), z["rec"])], Wave(c["T"], c["dt"], c["ddt"], c["f"]))[0]


@pytest.mark.parametrize("name", ["twolayer_split_nb32", "gradient_endonleft_nb40"])
def test_static_entry_matches_allocating_entry_twice(name):
    z, c, vp, rho = _case(name)
    ref = _allocating(z, c, vp, rho)
    for call in range(2):
        out = np.full(ref.size, np.nan, np.float32)
        rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], out)
        assert rc == 0, msg
        got = out.reshape(ref.shape)
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call}")
        assert O.rel_l2(got, z["seis"]) <= TOL


@pytest.mark.parametrize("where", ["model_device", "seis_device", "both_device"])
def test_static_entry_host_and_device_pointers(where):
    import torch
    from seis2d_b200 import _lib as L
    z, c, vp, rho = _case("edges_explicit_nb32")
    ref = _allocating(z, c, vp, rho).ravel()
    vp_d, rho_d = torch.from_numpy(vp).cuda(), torch.from_numpy(rho).cuda()
    out_d = torch.full((ref.size,), float("nan"), dtype=torch.float32, device="cuda")
    out_h = np.full(ref.size, np.nan, np.float32)
    flags, kw = 0, {}
    if where in ("model_device", "both_device"):
        flags |= L.S2D_STATIC_MODEL_DEVICE
        kw.update(vp_ptr=C.c_void_p(vp_d.data_ptr()), rho_ptr=C.c_void_p(rho_d.data_ptr()))
    if where in ("seis_device", "both_device"):
        flags |= L.S2D_STATIC_SEIS_DEVICE
        kw.update(out_ptr=C.c_void_p(out_d.data_ptr()))
    for call in range(2):
        rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], out_h, flags=flags, **kw)
        assert rc == 0, msg
        torch.cuda.synchronize()
        got = out_d.cpu().numpy() if flags & L.S2D_STATIC_SEIS_DEVICE else out_h
        np.testing.assert_array_equal(got, ref, err_msg=f"{where}, call {call}")


@pytest.mark.parametrize("flag", ["S2D_MODEL_FREE_SURFACE", "S2D_MODEL_ORDER8", "S2D_SEIS_DEVICE", "unknown"])
def test_static_entry_rejects_other_flags(flag):
    from seis2d_b200 import _lib as L
    z, c, vp, rho = _case("twolayer_split_nb32")
    bits = 0x4000 if flag == "unknown" else getattr(L, flag)
    out = np.zeros(z["seis"].size, np.float32)
    rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], out, flags=bits)
    assert rc == L.S2D_ERR_ARG, (rc, msg)
    assert "unsupported flag" in msg
    # the rejection leaves the entry usable
    rc, msg = _static_call(c, vp, rho, z["src"], z["rec"], out)
    assert rc == 0, msg


def test_static_entry_rejects_oversized_jobs():
    from seis2d_b200 import _lib as L
    z, c, vp, rho = _case("twolayer_split_nb32")
    big = dict(c, nx=3000, nz=3000)
    vpb = np.full((3000, 3000), 2000.0, np.float32)
    out = np.zeros(1, np.float32)
    rc, msg = _static_call(big, vpb, vpb, (100.0, 10.0), np.array([[10.0, 10.0]], np.float32), out)
    assert rc == L.S2D_ERR_NOMEM
    assert "needs" in msg and "static scratch holds" in msg
