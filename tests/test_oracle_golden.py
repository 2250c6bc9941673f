"""The CPU restatement (oracle/s2d_oracle.c) against the reference's own
outputs, stored in tests/golden/ by tests/golden/make_golden.py."""
import json

import numpy as np
import pytest

from cases import CASES, model
from oracle import oracle as O


def _load(name):
    z = np.load(f"{O.HERE}/../tests/golden/{name}.npz")
    c = json.loads(str(z["params"]))
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"])
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    return z, c, p, vp, rho


@pytest.mark.parametrize("name", sorted(CASES))
def test_f64_restatement_is_bit_exact(name):
    z, c, p, vp, rho = _load(name)
    rec = z["rec"]
    s = O.forward(p, vp, rho, z["src"], rec[:, 0], rec[:, 1], O.F64)
    assert s.shape == z["seis"].shape
    assert np.array_equal(s, z["seis"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_f32_restatement_within_tolerance(name):
    z, c, p, vp, rho = _load(name)
    rec = z["rec"]
    s = O.forward(p, vp, rho, z["src"], rec[:, 0], rec[:, 1], O.F32)
    # FP32 wavefields against the reference's FP64 ones: the 1e-5 bar.
    assert O.rel_l2(s, z["seis"]) < 1e-5


def test_derived_constants_match_reference_rules():
    # nts per the wavelet rule (cpumodelling.cpp:183-188) on the five
    # workload configurations: 15/20/20/15/10 Hz at 1/0.5/0.6/0.8/1 ms.
    got = []
    for f, dt, T in [(15, 0.001, 2.0), (20, 0.0005, 2.0), (20, 0.0006, 6.0), (15, 0.0008, 2.4), (10, 0.001, 3.0)]:
        d = O.derive(O.Params(100, 100, 40, 10.0, 10.0, T, dt, dt, f))
        got.append(d["nts"])
    assert got == [260, 390, 325, 325, 390]
    d = O.derive(O.Params(100, 100, 40, 10.0, 10.0, 2.4, 0.0008, 0.0008, 15))
    assert d["fd_nt"] == 3001  # float ceil of 2.4/0.0008


def test_ricker_peak_and_length():
    p = O.Params(50, 50, 32, 10.0, 10.0, 1.0, 0.001, 0.001, 15.0)
    w = O.ricker(p)
    assert w.size == O.derive(p)["nts"]
    t0 = 1.5 * np.sqrt(6.0) / (np.pi * 15.0)
    assert abs(np.argmax(w) * 0.001 - t0) < 0.001
    assert abs(w.max() - 1.0) < 1e-3
