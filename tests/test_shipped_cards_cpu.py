"""The reference's own two shipped job cards (input/sigsbee2a_3201x1201z.json,
input/twoLayer_model_5000x5000z.json) and the shot files they name
(geometry/*.json), read by the host driver, against the reference binary's
parse of them (json_parser.cpp:122-300), every shot's source and receivers as
it built them (create_geometry.cpp:237-444) and its stability verdicts
(check_stability.cpp:8-72) for velocity bounds on both sides of each limit.

The fixtures under tests/golden/shipped/ were written by
``tests/golden/make_golden.py --shipped`` (the cards copied as they are).  The
model files the cards name are not distributed; neither the parse, the
geometry nor the stability check reads them.  No GPU: host-only entry points.
"""
import json
import os
import shutil

import numpy as np
import pytest

from seis2d_b200 import driver as D
from seis2d_b200._lib import S2D_ERR_STABILITY, Seis2dError

SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "shipped")
CARDS = ["sigsbee2a_3201x1201z.json", "twoLayer_model_5000x5000z.json"]


def _dump(card):
    """The reference's parse and geometry of ``card`` (oracle/ref_harness.cpp --dump-job)."""
    lines = open(os.path.join(SHIPPED, card.replace(".json", ".dump.txt"))).read().splitlines()
    kv, shots, i = {}, [], 0
    while not lines[i].startswith("nsrc"):
        k, _, v = lines[i].partition(" ")
        kv[k] = v
        i += 1
    nsrc = int(lines[i].split()[1])
    i += 1
    for _ in range(nsrc):
        _, _, sx, sz, n = lines[i].split()
        rec = np.array([[float(t) for t in l.split()] for l in lines[i + 1:i + 1 + int(n)]], np.float32).reshape(-1, 2)
        shots.append(((np.float32(sx), np.float32(sz)), rec))
        i += 1 + int(n)
    return kv, shots


@pytest.fixture
def layout(tmp_path, monkeypatch):
    """The cards' relative layout: cwd input/, shot files in ../geometry/."""
    for sub in ("input", "geometry"):
        shutil.copytree(os.path.join(SHIPPED, sub), tmp_path / sub)
    monkeypatch.chdir(tmp_path / "input")
    return tmp_path


@pytest.mark.parametrize("card", CARDS)
def test_shipped_card_parse(layout, card):
    kv, _ = _dump(card)
    c = D.read_jobcard(card)
    assert c.velfile.decode() == kv["velfile"] and c.densfile.decode() == kv["densfile"]
    assert (c.nx, c.nz) == (int(kv["nx"]), int(kv["nz"]))
    assert (c.dx, c.dz) == (np.float32(kv["dx"]), np.float32(kv["dz"]))
    w = c.wave
    assert (w.rec_len, w.fd_dt, w.real_dt, w.dom_freq) == tuple(
        np.float32(kv[k]) for k in ("rec_len", "fd_dt", "real_dt", "dom_freq"))
    assert (c.geomflag, c.fdop, c.frsf) == (int(kv["geomflag"]), int(kv["fdop"]), int(kv["frsf"]))
    assert c.jbtype.decode() == kv["jbtype"]
    assert c.jobname.decode() == kv["jobname"] and c.tmppath.decode() == kv["tmppath"]


@pytest.mark.parametrize("card", CARDS)
def test_shipped_card_geometry_every_shot(layout, card):
    _, ref = _dump(card)
    got = D.read_geometry(D.read_jobcard(card))
    assert len(got) == len(ref)
    for s, ((src, rec), (rsrc, rrec)) in enumerate(zip(got, ref)):
        assert (np.float32(src[0]), np.float32(src[1])) == rsrc, s
        assert rec.shape == rrec.shape, s
        np.testing.assert_array_equal(rec, rrec, err_msg=f"shot {s}")


@pytest.mark.parametrize("card", CARDS)
def test_shipped_card_stability_verdicts(layout, card):
    verdicts = json.load(open(os.path.join(SHIPPED, "stability.json")))[card]
    c = D.read_jobcard(card)
    for v in verdicts:
        if v["stable"]:
            D.check_stability(c, v["vmin"], v["vmax"])
        else:
            assert v["exit"] == (-5) & 0xFF  # MPI::COMM_WORLD.Abort(-5)
            with pytest.raises(Seis2dError) as e:
                D.check_stability(c, v["vmin"], v["vmax"])
            assert e.value.code == S2D_ERR_STABILITY and "reference code -5" in str(e.value)
