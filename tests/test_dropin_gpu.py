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
