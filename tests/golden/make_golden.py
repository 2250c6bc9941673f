"""Generate the golden seismograms in tests/golden/ from the reference itself.

Runs the reference CPU binary (SeisAcoMod2D src/src_cpu, built unmodified by
``make -C oracle ref`` and, for other sponge widths, ``make -C oracle ref
NB=<nb>`` whose only change is the npml constant) on each case of
``cases.py`` and stores, per case, ``<case>.npz`` with:

  seis      float32 [nrec][real_nt]  the reference's output file
  src       float32 (2,)             source (x, z) metres (from test_geometry.txt)
  rec       float32 (nrec, 2)        receivers (x, z) metres, as the reference built them
  params    json                     the run parameters
  jobcard   text                     the job card the reference read
  geomfile  text                     the shot or geometry file it read

Needs the reference tree (to build the binary), so it runs in the development
container; the committed .npz files are what the tests use everywhere.
Usage: python tests/golden/make_golden.py [case ...]
       python tests/golden/make_golden.py --geometry   (geometry_cases.json)
       python tests/golden/make_golden.py --shipped    (shipped/: the reference's
           own two job cards and shot files, copied as they are, with the
           reference binary's parse, every shot's geometry and its stability
           verdicts for a few velocity bounds; the model files those cards
           name are not distributed, and the parse and geometry need none)
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, explicit_geometry, model  # noqa: E402
from seis2d_b200 import formats as F  # noqa: E402


def _ref_root():
    """SeisAcoMod2D checkout: $SEISACOMOD2D_REF, else ``reference`` beside the repository."""
    return os.environ.get("SEISACOMOD2D_REF") or os.path.join(os.path.dirname(ROOT), "reference")


def _make_ref(nb=32):
    args = ["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
            f"REF_SRC={os.path.join(_ref_root(), 'src', 'src_cpu')}"]
    if nb != 32:
        args.append(f"NB={nb}")
    subprocess.run(args, check=True)


def run_case(name: str, c: dict) -> dict:
    nb = c["nb"]
    binary = os.path.join(ROOT, "oracle", "_ref", "seis_ref" if nb == 32 else f"seis_ref_nb{nb}")
    _make_ref(nb)
    vp, rho = model(c["model"], c["nx"], c["nz"], c["dx"], c["dz"])
    with tempfile.TemporaryDirectory() as wd:
        F.write_model(os.path.join(wd, "vp.bin"), vp)
        F.write_model(os.path.join(wd, "rho.bin"), rho)
        kind, spec = c["geom"]
        card = {
            "Velocity": "vp.bin", "Density": "rho.bin", "NX": c["nx"], "NZ": c["nz"],
            "DX": c["dx"], "DZ": c["dz"], "Time": c["T"], "FD DT": c["dt"], "DATA DT": c["ddt"],
            "Frequency": c["f"], "Output Directory": "out", "Free surface": 0,
            "Job type New or Restart": "New", "Order of FD Operator": 4,
        }
        if kind == "shot":
            F.write_shotfile(os.path.join(wd, "geom.txt"), spec)
            card.update({"Read source receiver flag": 1, "if choice=0, Geometry file": "NA",
                         "if choice=1, Shot file": "geom.txt"})
        else:
            F.write_geometry(os.path.join(wd, "geom.txt"),
                             explicit_geometry(spec, c["nx"], c["nz"], c["dx"], c["dz"]))
            card.update({"Read source receiver flag": 0, "if choice=0, Geometry file": "geom.txt",
                         "if choice=1, Shot file": "NA"})
        F.write_jobcard(os.path.join(wd, "case.json"), card)
        os.makedirs(os.path.join(wd, "out"))
        r = subprocess.run([binary, "case.json"], cwd=wd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        g = np.loadtxt(os.path.join(wd, "test_geometry.txt"), dtype=np.float64, ndmin=2)
        src = np.array([g[0, 1], g[0, 0]], np.float32)
        rec = np.stack([g[1:, 1], g[1:, 0]], axis=1).astype(np.float32)
        seis = F.read_seismogram(os.path.join(wd, "out", "case_seismogram.bin"), rec.shape[0])
        jobcard = open(os.path.join(wd, "case.json")).read()
        geomfile = open(os.path.join(wd, "geom.txt")).read()
    params = dict(c)
    params.pop("geom")
    params["geom_kind"] = kind
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, seis=seis, src=src, rec=rec, params=json.dumps(params),
                        jobcard=jobcard, geomfile=geomfile)
    return {"case": name, "nrec": int(rec.shape[0]), "nt": int(seis.shape[1]),
            "max_abs": float(np.abs(seis).max()), "bytes": os.path.getsize(out)}


# Shot-file spreads whose receiver lists the reference builds
# (create_geometry.cpp:237-444), each run as a one-shot job of one FD step so
# that print_single_source_geometry (create_geometry.cpp:446-459) writes them.
# Split spreads with a near offset are left out: the reference writes one
# receiver past the end of its array for every such shot.
GEOMETRY_CASES = [
    # (nx, nz, dx, dz, sx, sz, nrec, nearoff, spacing, type)
    (200, 40, 10.0, 10.0, 1000.0, 20.0, 81, 0, 10.0, 1),     # split, room on both sides
    (200, 40, 10.0, 10.0, 100.0, 20.0, 80, 0, 10.0, 1),      # split, short on the left
    (200, 40, 10.0, 10.0, 1900.0, 0.0, 80, 0, 20.0, 1),      # split, short on the right
    (200, 40, 10.0, 10.0, 1500.0, 10.0, 100, 0, 10.0, 2),    # end-on left
    (200, 40, 10.0, 10.0, 1500.0, 10.0, 60, 30.0, 20.0, 2),  # end-on left, near offset
    (200, 40, 10.0, 10.0, 200.0, 30.0, 120, 0, 10.0, 3),     # end-on right
    (200, 40, 10.0, 10.0, 200.0, 30.0, 50, 10.0, 30.0, 3),   # end-on right, near offset
    (600, 40, 7.62, 7.62, 2286.0, 15.24, 101, 0, 15.24, 1),  # non-integer spacing (float drift)
    (600, 40, 7.62, 7.62, 3048.0, 7.62, 151, 0, 7.62, 2),
    (600, 40, 7.62, 7.62, 762.0, 0.0, 151, 0, 22.86, 3),
]


def run_geometry_cases():
    _make_ref()
    binary = os.path.join(ROOT, "oracle", "_ref", "seis_ref")
    out = []
    for (nx, nz, dx, dz, sx, sz, nrec, near, sp, gt) in GEOMETRY_CASES:
        with tempfile.TemporaryDirectory() as wd:
            m = np.full((nx, nz), 2000.0, np.float32)
            F.write_model(os.path.join(wd, "vp.bin"), m)
            F.write_model(os.path.join(wd, "rho.bin"), m)
            F.write_shotfile(os.path.join(wd, "shots.txt"), [(sx, sz, nrec, near, sp, gt)])
            F.write_jobcard(os.path.join(wd, "g.json"), {
                "Velocity": "vp.bin", "Density": "rho.bin", "NX": nx, "NZ": nz, "DX": dx, "DZ": dz,
                "Time": 0.001, "FD DT": 0.001, "DATA DT": 0.001, "Frequency": 5.0,
                "Read source receiver flag": 1, "if choice=0, Geometry file": "NA",
                "if choice=1, Shot file": "shots.txt", "Output Directory": "out", "Free surface": 0,
                "Job type New or Restart": "New", "Order of FD Operator": 4})
            os.makedirs(os.path.join(wd, "out"))
            r = subprocess.run([binary, "--no-stability", "g.json"], cwd=wd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"geometry case {sx},{gt}: reference exited {r.returncode}")
            shotfile = open(os.path.join(wd, "shots.txt")).read()
            printed = open(os.path.join(wd, "test_geometry.txt")).read()
        out.append({"nx": nx, "nz": nz, "dx": dx, "dz": dz, "shotfile": shotfile, "test_geometry": printed})
    with open(os.path.join(HERE, "geometry_cases.json"), "w") as f:
        json.dump(out, f, indent=0)
    return len(out)


# The reference's shipped cards (input/*.json) and the shot files they name
# (geometry/*.json), and velocity bounds (vmin, vmax) around each card's
# stability (dt <= 0.606 h_min / v_max) and dispersion (2 f <= v_min / (5 h_max))
# limits: check_stability.cpp:8-72.
SHIPPED = {
    "sigsbee2a_3201x1201z.json": [(1500.0, 4500.0), (1500.0, 4700.0), (1300.0, 4500.0), (1371.0, 4600.0)],
    "twoLayer_model_5000x5000z.json": [(1500.0, 3000.0), (1499.0, 3000.0), (2000.0, 6100.0), (1500.0, 6060.0)],
}


def run_shipped(ref_root):
    import shutil
    _make_ref()
    binary = os.path.join(ROOT, "oracle", "_ref", "seis_ref")
    dest = os.path.join(HERE, "shipped")
    for sub in ("input", "geometry"):
        os.makedirs(os.path.join(dest, sub), exist_ok=True)
    out = {}
    for card, bounds in SHIPPED.items():
        shutil.copyfile(os.path.join(ref_root, "input", card), os.path.join(dest, "input", card))
        text = open(os.path.join(dest, "input", card)).read()
        shotfile = [l.split(":", 1)[1].strip().strip('"') for l in text.splitlines() if "Shot file" in l][0]
        shutil.copyfile(os.path.join(ref_root, "input", shotfile), os.path.join(dest, "input", shotfile))
        verdicts = []
        with tempfile.TemporaryDirectory() as wd:
            for sub in ("input", "geometry"):
                shutil.copytree(os.path.join(dest, sub), os.path.join(wd, sub))
            cwd = os.path.join(wd, "input")
            r = subprocess.run([binary, "--dump-job", "dump.txt", card], cwd=cwd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"{card}: reference exited {r.returncode}\n{r.stdout[-2000:]}")
            dump = open(os.path.join(cwd, "dump.txt")).read()
            for vmin, vmax in bounds:
                r = subprocess.run([binary, "--dump-job", "chk.txt", "--check", repr(vmin), repr(vmax), card],
                                   cwd=cwd, capture_output=True, text=True)
                stable = r.returncode == 0 and open(os.path.join(cwd, "chk.txt")).read().endswith("STABLE\n")
                verdicts.append({"vmin": vmin, "vmax": vmax, "stable": stable, "exit": r.returncode})
        with open(os.path.join(dest, card.replace(".json", ".dump.txt")), "w") as f:
            f.write(dump)
        out[card] = verdicts
    with open(os.path.join(dest, "stability.json"), "w") as f:
        json.dump(out, f, indent=1)
    return {k: len(v) for k, v in out.items()}


def main(argv):
    if argv[:1] == ["--shipped"]:
        print(json.dumps(run_shipped(argv[1] if len(argv) > 1 else _ref_root())))
        return
    if argv == ["--geometry"]:
        print(json.dumps({"geometry_cases": run_geometry_cases()}))
        return
    names = argv or list(CASES)
    for n in names:
        print(json.dumps(run_case(n, CASES[n])))


if __name__ == "__main__":
    main(sys.argv[1:])
