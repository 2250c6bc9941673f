"""The drop-in build (oracle/_ref/seis_dropin: the reference's own host program
linked with seis2d_b200/integration/modelling_module_b200.cpp and libseis2d)
on a machine without a GPU: the reference's job-card, geometry, model and
stability code run unchanged and hand the shots to the B200 modelling_module,
which stops with the binding's code -20 because no CUDA device is usable."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "seis_dropin")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def stage(tmp, name):
    from cases import model
    from seis2d_b200 import formats as F
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    F.write_model(str(tmp / "vp.bin"), vp)
    F.write_model(str(tmp / "rho.bin"), rho)
    (tmp / "case.json").write_text(str(z["jobcard"]))
    (tmp / "geom.txt").write_text(str(z["geomfile"]))
    os.makedirs(tmp / "out", exist_ok=True)
    return z, c


def test_dropin_reaches_modelling_module_without_gpu(tmp_path):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/seis_dropin not built (needs the reference sources: make -C oracle dropin)")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: tests/test_dropin_gpu.py covers the drop-in there")
    z, c = stage(tmp_path, "edges_explicit_nb32")
    r = subprocess.run([DROPIN, "case.json"], cwd=tmp_path, capture_output=True, text=True,
                       env=dict(os.environ, S2D_NB=str(c["nb"])))
    assert r.returncode == (-20) & 0xFF, r.stderr
    assert "no usable CUDA device" in r.stderr
    # the reference's master ran first: geometry and workload were printed by its own code
    assert "Job file" in r.stdout
