"""Whole jobs from job cards (s2d_run_jobcard and the seis2d_run command):
the seismogram files must match the reference's files for the same card."""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from seis2d_b200 import driver as D
from seis2d_b200 import formats as F

pytestmark = pytest.mark.gpu

TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _stage(tmp, name):
    from cases import model
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = json.loads(str(z["params"]))
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    F.write_model(str(tmp / "vp.bin"), vp)
    F.write_model(str(tmp / "rho.bin"), rho)
    (tmp / "case.json").write_text(str(z["jobcard"]))
    (tmp / "geom.txt").write_text(str(z["geomfile"]))
    os.makedirs(tmp / "out", exist_ok=True)
    return z, c


@pytest.mark.parametrize("name", ["twolayer_split_nb32", "gradient_endonleft_nb40", "edges_explicit_nb32"])
def test_run_jobcard_matches_reference_file(tmp_path, monkeypatch, name):
    monkeypatch.chdir(tmp_path)
    z, c = _stage(tmp_path, name)
    D.run_jobcard("case.json", nb=c["nb"], naming="cpu")
    got = F.read_seismogram("out/case_seismogram.bin", z["rec"].shape[0])
    assert got.shape == z["seis"].shape
    assert O.rel_l2(got, z["seis"]) <= TOL


def test_gpu_naming_and_restart(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    z, c = _stage(tmp_path, "twolayer_split_nb32")
    F.write_shotfile("geom.txt", [(300.0, 20.0, 41, 0, 10.0, 1), (800.0, 20.0, 41, 0, 10.0, 1),
                                  (1200.0, 20.0, 41, 0, 10.0, 1)])
    D.run_jobcard("case.json", nb=c["nb"], naming="gpu")
    names = sorted(os.listdir("out"))
    assert names == ["case_checkpoint_rank0.txt", "case_sx1200.00_seismogram.bin", "case_sx300.00_seismogram.bin",
                     "case_sx800.00_seismogram.bin"]
    assert open("out/case_checkpoint_rank0.txt").read().strip() == "3"
    first = {n: open("out/" + n, "rb").read() for n in names if n.endswith(".bin")}
    # restart after the second shot: only the third is modelled again
    for n in first:
        os.remove("out/" + n)
    open("out/case_checkpoint_rank0.txt", "w").write("2\n")
    (tmp_path / "case.json").write_text(str(z["jobcard"]).replace('"New"', '"Restart"'))
    D.run_jobcard("case.json", nb=c["nb"], naming="gpu")
    assert sorted(n for n in os.listdir("out") if n.endswith(".bin")) == ["case_sx1200.00_seismogram.bin"]
    assert open("out/case_sx1200.00_seismogram.bin", "rb").read() == first["case_sx1200.00_seismogram.bin"]


def test_command_line_driver(tmp_path):
    z, c = _stage(tmp_path, "layers_endonright_near_nb32")
    exe = os.path.join(ROOT, "seis2d_b200", "bin", "seis2d_run")
    r = subprocess.run([exe, "--quiet", "--nb", str(c["nb"]), "case.json"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    got = F.read_seismogram(str(tmp_path / "out" / "case_seismogram.bin"), z["rec"].shape[0])
    assert O.rel_l2(got, z["seis"]) <= TOL
    # a card that fails the stability rule stops with the reference's code in the message
    (tmp_path / "case.json").write_text(str(z["jobcard"]).replace('"0.001"', '"0.004"', 1))
    r = subprocess.run([exe, "--quiet", "case.json"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "reference code -" in r.stderr


def test_ranks_of_a_job_write_the_whole_jobs_files(tmp_path, monkeypatch):
    """The ranks of a 2-rank job (run one after the other on one GPU; they
    never wait on each other) together write the files of the 1-rank job,
    each rank keeping its own restart index of its block."""
    monkeypatch.chdir(tmp_path)
    z, c = _stage(tmp_path, "twolayer_split_nb32")
    shots = [(200.0 + 150.0 * k, 20.0, 31, 0, 10.0, 1) for k in range(5)]
    F.write_shotfile("geom.txt", shots)
    D.run_jobcard("case.json", nb=c["nb"], naming="gpu")
    whole = {n: open("out/" + n, "rb").read() for n in os.listdir("out") if n.endswith(".bin")}
    assert len(whole) == 5
    for n in os.listdir("out"):
        os.remove("out/" + n)
    for rank in (0, 1):
        D.run_jobcard("case.json", nb=c["nb"], naming="gpu", rank=rank, nranks=2)
    got = {n: open("out/" + n, "rb").read() for n in os.listdir("out") if n.endswith(".bin")}
    assert got == whole
    assert open("out/case_checkpoint_rank0.txt").read().strip() == "3"
    assert open("out/case_checkpoint_rank1.txt").read().strip() == "2"
    # restart of rank 1 after its first shot: only the last shot runs again
    os.remove("out/case_sx800.00_seismogram.bin")
    os.remove("out/case_sx500.00_seismogram.bin")
    open("out/case_checkpoint_rank1.txt", "w").write("1\n")
    (tmp_path / "case.json").write_text(str(z["jobcard"]).replace('"New"', '"Restart"'))
    D.run_jobcard("case.json", nb=c["nb"], naming="gpu", rank=1, nranks=2)
    assert os.path.exists("out/case_sx800.00_seismogram.bin")
    assert not os.path.exists("out/case_sx500.00_seismogram.bin")
    assert open("out/case_sx800.00_seismogram.bin", "rb").read() == whole["case_sx800.00_seismogram.bin"]
