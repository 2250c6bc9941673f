"""C ABI checks that need no GPU: the library loads, exports every symbol the
public headers declare, and its host-only entry points agree with the
oracle's derivation of the run constants."""
import ctypes as C
import glob
import os
import re

import pytest

from oracle import oracle as O
from seis2d_b200 import _lib as L
from seis2d_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"S2D_API\s+[^;(]*?\b(s2d_\w+)\s*\(", txt))
    return names


def test_library_builds_and_loads():
    B.build()
    assert os.path.exists(L.LIB_PATH)
    assert L.lib().s2d_abi_version() == 3


def test_every_declared_symbol_is_exported():
    declared = _declared_symbols()
    assert {"s2d_create", "s2d_forward", "s2d_model_create"} <= declared
    lib = C.CDLL(L.LIB_PATH)
    for name in declared:
        assert hasattr(lib, name), name
    assert declared <= set(L.SIGNATURES) | declared  # every binding known to the wrapper
    assert set(L.SIGNATURES) <= declared


@pytest.mark.parametrize("T,dt,ddt,f", [(2.0, 0.001, 0.001, 15.0), (2.0, 0.0005, 0.0005, 20.0),
                                        (6.0, 0.0006, 0.0006, 20.0), (2.4, 0.0008, 0.0008, 15.0),
                                        (3.0, 0.001, 0.004, 10.0), (0.5, 0.0008, 0.0016, 10.0)])
def test_derive_steps_matches_oracle(T, dt, ddt, f):
    from seis2d_b200 import Wave, derive_steps
    got = derive_steps(Wave(T, dt, ddt, f))
    want = O.derive(O.Params(10, 10, 32, 10.0, 10.0, T, dt, ddt, f))
    for k in ("fd_nt", "real_nt", "dt_factor", "nts"):
        assert got[k] == want[k], k


def test_bad_wave_rejected():
    st = L.Steps()
    assert L.lib().s2d_derive_steps(C.byref(L.Wave(1.0, 0.0, 0.001, 10.0)), C.byref(st)) == L.S2D_ERR_ARG
    assert L.lib().s2d_derive_steps(None, C.byref(st)) == L.S2D_ERR_ARG


def test_null_context_is_an_error_not_a_crash():
    assert L.lib().s2d_model_destroy(None, 1) == L.S2D_ERR_ARG
    assert L.lib().s2d_forward(None, None, 0, None, None, 0, 0, 0, None, 0, None) == L.S2D_ERR_ARG
    assert L.lib().s2d_last_error(None) == b"null context"


def test_no_device_reports_nodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert L.lib().s2d_create(C.byref(h), 0) == L.S2D_ERR_NODEV
