"""Host driver (job card, geometry, stability) against the reference's own
behaviour.  No GPU: these entry points are host-only.

Receiver lists are compared as the text the reference prints for a shot
(print_single_source_geometry, create_geometry.cpp:446-459, "%f %f" of z, x),
captured from the reference binary in tests/golden/geometry_cases.json and the
golden .npz files."""
import json
import os

import numpy as np
import pytest

from seis2d_b200 import driver as D
from seis2d_b200 import formats as F
from seis2d_b200._lib import (S2D_ERR_GEOM, S2D_ERR_IO, S2D_ERR_JOBCARD, S2D_ERR_STABILITY, Seis2dError)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BASE = {"Velocity": "vp.bin", "Density": "rho.bin", "NX": 200, "NZ": 40, "DX": 10.0, "DZ": 10.0,
        "Time": 0.5, "FD DT": 0.001, "DATA DT": 0.002, "Frequency": 10.0, "Read source receiver flag": 1,
        "if choice=0, Geometry file": "NA", "if choice=1, Shot file": "shots.txt", "Output Directory": "out",
        "Free surface": 0, "Job type New or Restart": "New", "Order of FD Operator": 4}


def _printed(src, rec):
    lines = ["%f %f" % (np.float32(src[1]), np.float32(src[0]))]
    lines += ["%f %f" % (np.float32(z), np.float32(x)) for x, z in rec]
    return "\n".join(lines) + "\n"


def _card(tmp_path, **over):
    p = dict(BASE)
    p.update(over)
    path = str(tmp_path / "job.json")
    F.write_jobcard(path, p)
    return path


@pytest.fixture
def in_tmp(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    return tmp_path


def test_geometry_cases_match_reference_printout(in_tmp):
    cases = json.load(open(os.path.join(GOLDEN, "geometry_cases.json")))
    for c in cases:
        (in_tmp / "shots.txt").write_text(c["shotfile"])
        card = D.read_jobcard(_card(in_tmp, NX=c["nx"], NZ=c["nz"], DX=c["dx"], DZ=c["dz"]))
        [(src, rec)] = D.read_geometry(card)
        assert _printed(src, rec) == c["test_geometry"], c["shotfile"]


@pytest.mark.parametrize("name", ["twolayer_split_nb32", "gradient_endonleft_nb40", "layers_endonright_near_nb32",
                                  "edges_explicit_nb32", "corner_source_nb40"])
def test_golden_cards_and_geometry(in_tmp, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = json.loads(str(z["params"]))
    (in_tmp / "case.json").write_text(str(z["jobcard"]))
    (in_tmp / "geom.txt").write_text(str(z["geomfile"]))
    card = D.read_jobcard("case.json")
    assert (card.nx, card.nz, card.dx, card.dz) == (c["nx"], c["nz"], np.float32(c["dx"]), np.float32(c["dz"]))
    assert card.wave.fd_dt == np.float32(c["dt"]) and card.wave.real_dt == np.float32(c["ddt"])
    assert card.jobname == b"case_" and card.tmppath == b"out/" and card.fdop == 4
    [(src, rec)] = D.read_geometry(card)
    assert tuple(np.float32(src)) == tuple(z["src"])
    assert np.array_equal(rec, z["rec"])


def test_explicit_geometry_groups_shots(in_tmp):
    rows = []
    for sx in (100.0, 300.0, 500.0):
        for gx in range(0, 200, 20):
            rows.append(f"{sx:f},10.000000,{gx * 10.0:f},20.000000")
    (in_tmp / "g.txt").write_text("\n".join(rows) + "\n")
    card = D.read_jobcard(_card(in_tmp, **{"Read source receiver flag": 0, "if choice=0, Geometry file": "g.txt"}))
    g = D.read_geometry(card)
    assert [s for s, _ in g] == [(100.0, 10.0), (300.0, 10.0), (500.0, 10.0)]
    assert all(r.shape == (10, 2) for _, r in g)
    assert g[1][1][3].tolist() == [600.0, 20.0]


def test_jobname_and_output_dir(in_tmp):
    os.makedirs(in_tmp / "cards")
    F.write_jobcard(str(in_tmp / "cards" / "my.card.json"), dict(BASE, **{"Output Directory": "res/"}))
    card = D.read_jobcard(str(in_tmp / "cards" / "my.card.json"))
    assert card.jobname == b"my.card_" and card.tmppath == b"res/"


def test_first_occurrence_of_a_key_wins_and_comments_skipped(in_tmp):
    path = _card(in_tmp)
    with open(path, "a") as f:
        f.write('    "NX" : "999"\n"comment" : "NX 5"\n')
    assert D.read_jobcard(path).nx == 200


@pytest.mark.parametrize("key", ["Velocity", "Density", "NX", "NZ", "DX", "DZ", "Time", "FD DT", "DATA DT",
                                 "Frequency", "Read source receiver flag", "if choice=1, Shot file",
                                 "Output Directory", "Free surface", "Job type New or Restart",
                                 "Order of FD Operator"])
def test_missing_key_is_a_jobcard_error(in_tmp, key):
    p = dict(BASE)
    p.pop(key)
    path = str(in_tmp / "job.json")
    F.write_jobcard(path, p)
    with pytest.raises(Seis2dError) as e:
        D.read_jobcard(path)
    assert e.value.code == S2D_ERR_JOBCARD and "reference code -6" in str(e.value)


@pytest.mark.parametrize("over", [{"DATA DT": 0.0015}, {"Read source receiver flag": 2}, {"Free surface": 3},
                                  {"Job type New or Restart": "new"}, {"NX": "abc"}])
def test_bad_values_are_jobcard_errors(in_tmp, over):
    with pytest.raises(Seis2dError) as e:
        D.read_jobcard(_card(in_tmp, **over))
    assert e.value.code == S2D_ERR_JOBCARD


def test_missing_card_is_io_error(in_tmp):
    with pytest.raises(Seis2dError) as e:
        D.read_jobcard("nope.json")
    assert e.value.code == S2D_ERR_IO


@pytest.mark.parametrize("line,code", [
    ("1000.0,20.0,81,0,10.0", "-25"),        # five fields
    ("1000.0,20.0,0,0,10.0,1", "-18"),       # no receivers
    ("1005.0,20.0,81,0,10.0,1", "-13"),      # source off the grid
    ("1000.0,25.0,81,0,10.0,1", "-14"),
    ("1000.0,20.0,81,0,15.0,1", "-15"),      # spacing off the grid
    ("5000.0,20.0,81,0,10.0,1", "-16"),      # source outside the model
    ("100.0,20.0,81,0,10.0,2", "-3"),        # end-on-left spread leaves the model
    ("1000.0,20.0,81,0,10.0,4", "-12"),      # unknown spread type
    ("1000.0,20.0,81,0,10.0,1\n1200.0,20.0,81,0,10.0,2", "-11"),  # mixed spread types
])
def test_shot_file_errors(in_tmp, line, code):
    (in_tmp / "shots.txt").write_text(line + "\n")
    card = D.read_jobcard(_card(in_tmp))
    with pytest.raises(Seis2dError) as e:
        D.read_geometry(card)
    assert e.value.code == S2D_ERR_GEOM and f"reference code {code})" in str(e.value)


def test_unsorted_explicit_geometry_rejected(in_tmp):
    (in_tmp / "g.txt").write_text("300.0,10.0,0.0,20.0\n100.0,10.0,0.0,20.0\n")
    card = D.read_jobcard(_card(in_tmp, **{"Read source receiver flag": 0, "if choice=0, Geometry file": "g.txt"}))
    with pytest.raises(Seis2dError) as e:
        D.read_geometry(card)
    assert "reference code -22" in str(e.value)


def test_stability_and_dispersion_checks(in_tmp):
    card = D.read_jobcard(_card(in_tmp))
    D.check_stability(card, 1500.0, 3000.0)
    with pytest.raises(Seis2dError) as e:  # dt 1 ms > 0.606 * 10 / 7000
        D.check_stability(card, 1500.0, 7000.0)
    assert e.value.code == S2D_ERR_STABILITY
    # the 3201x1201 / 7.62 m / 20 Hz configuration fails the dispersion rule by 2%
    c3 = D.read_jobcard(_card(in_tmp, NX=3201, NZ=1201, DX=7.62, DZ=7.62, Frequency=20.0, **{"FD DT": 0.0006,
                                                                                            "DATA DT": 0.0006}))
    with pytest.raises(Seis2dError) as e:
        D.check_stability(c3, 1500.0, 4500.0)
    assert e.value.code == S2D_ERR_STABILITY and "dispersion" in str(e.value)


def test_fd_order_rules(in_tmp):
    """Order 8 (the 8th-order operator) has the tighter stability bound
    0.549 h / vmax; orders other than 4 and 8 stop the job before any device
    work (the reference parses the key and steps only for 4)."""
    c8 = D.read_jobcard(_card(in_tmp, **{"Order of FD Operator": 8}))
    assert c8.fdop == 8
    c4 = D.read_jobcard(_card(in_tmp))
    D.check_stability(c4, 1500.0, 5800.0)  # 1 ms <= 0.606 * 10 / 5800
    with pytest.raises(Seis2dError) as e:  # 1 ms > 0.549 * 10 / 5800
        D.check_stability(c8, 1500.0, 5800.0)
    assert e.value.code == S2D_ERR_STABILITY
    D.check_stability(c8, 1500.0, 5400.0)
    path = _card(in_tmp, **{"Order of FD Operator": 6})
    with pytest.raises(Seis2dError) as e:
        D.run_jobcard(path)
    assert e.value.code == S2D_ERR_JOBCARD and "order" in str(e.value)
