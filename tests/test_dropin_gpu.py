"""The drop-in build on a GPU: the reference's own host program (main,
Modelling_master, job card, geometry, model, stability code, unmodified)
linked with seis2d_b200/integration/modelling_module_b200.cpp and libseis2d
in place of cpumodelling.o writes, for every golden job card, the seismogram
file the reference CPU backend wrote (rel-L2 <= 1e-5)."""
import os
import subprocess

import pytest

from oracle import oracle as O
from seis2d_b200 import formats as F

from test_dropin_cpu import DROPIN, stage

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("name", ["twolayer_split_nb32", "gradient_endonleft_nb40", "edges_explicit_nb32",
                                  "layers_endonright_near_nb32", "corner_source_nb40", "salt_grid_nb50",
                                  "twolayer_5m_nb60"])
def test_dropin_writes_the_reference_file(tmp_path, name):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/seis_dropin not built")
    z, c = stage(tmp_path, name)
    r = subprocess.run([DROPIN, "case.json"], cwd=tmp_path, capture_output=True, text=True,
                       env=dict(os.environ, S2D_NB=str(c["nb"])))
    assert r.returncode == 0, r.stderr[-2000:]
    got = F.read_seismogram(str(tmp_path / "out" / "case_seismogram.bin"), z["rec"].shape[0])
    assert got.shape == z["seis"].shape
    assert O.rel_l2(got, z["seis"]) <= TOL


@pytest.mark.parametrize("key,value,fs,order", [("Free surface", "1", 1, 4), ("Order of FD Operator", "8", 0, 8)])
def test_dropin_honours_free_surface_and_order8(tmp_path, key, value, fs, order):
    """Keys the reference parses and ignores: through its own host program the
    drop-in gives the oracle's traces for the free surface and the 8th-order
    operator (no reference output exists for them)."""
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/seis_dropin not built")
    from cases import model
    z, c = stage(tmp_path, "twolayer_split_nb32")
    card = (tmp_path / "case.json").read_text()
    old = f'"{key}" : "0"' if key == "Free surface" else f'"{key}" : "4"'
    assert old in card
    (tmp_path / "case.json").write_text(card.replace(old, f'"{key}" : "{value}"'))
    r = subprocess.run([DROPIN, "case.json"], cwd=tmp_path, capture_output=True, text=True,
                       env=dict(os.environ, S2D_NB=str(c["nb"])))
    assert r.returncode == 0, r.stderr[-2000:]
    got = F.read_seismogram(str(tmp_path / "out" / "case_seismogram.bin"), z["rec"].shape[0])
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    p = O.Params(c["nx"], c["nz"], c["nb"], c["dx"], c["dz"], c["T"], c["dt"], c["ddt"], c["f"], fs, order)
    ref = O.forward(p, vp, rho, z["src"], z["rec"][:, 0], z["rec"][:, 1], O.F64)
    assert O.rel_l2(got, ref) <= TOL
    assert O.rel_l2(got, z["seis"]) > 1e-3
