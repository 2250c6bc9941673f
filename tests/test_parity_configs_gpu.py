"""Seismogram parity at the five workload configurations, at their full step
counts, against the reference's own CPU path.

For each configuration one shot (one per model for the uneven batch) is run
through the C ABI (s2d_forward) and by the reference binary
(oracle/_ref/seis_ref_nbNN: SeisAcoMod2D src/src_cpu built unmodified apart
from the sponge width; its time loop is src/src_cpu/cpumodelling.cpp:326-380)
on the same seeded synthetic model and the same explicit geometry, and the
traces must agree within rel-L2 1e-5.  The reference's wavefields are FP64 and
its output is their float32 rounding, so the same number is the error of the
FP32 kernels against an FP64 run of the scheme (the oracle's FP64
restatement, oracle/s2d_oracle.c, is bit-exact with that binary).

The error is also reported as it grows with the record length: rel-L2 over
the first quarter, half, three quarters and all of the samples
(``-s`` prints one PARITY line per configuration; S2D_PARITY_JSON=<path>
appends them to a file).

Configurations (models from bench.py's seeded generators):
  c1  two-layer 1000 x 1000, nb 40, 15 Hz, dt 1 ms, 2000 steps, 1000 receivers
  c2  two-layer 5000 x 5000, nb 60, 20 Hz, dt 0.5 ms, first 1000 of its 4000
      steps (0.5 s; the reference needs about a minute per 1000 steps of this
      grid on 16 host cores), 5000 receivers, the first of its 64 shots
  c3  salt 3201 x 1201, d 7.62 m, nb 50, 20 Hz, dt 0.6 ms, all 10000 steps,
      3201 receivers (the reference's dispersion check fails this grid by 2%,
      so both runs skip it)
  c4  601 x 301, 1201 x 601 and 2401 x 801 layered models, nb 50, 15 Hz,
      dt 0.8 ms, 3000 steps, one shot per model, the three in ONE batched call
  c5  1201 x 401 true FWI model, nb 50, 10 Hz, dt 1 ms, 3000 steps, 1201
      receivers, the middle of its 32 shots
"""
import json
import os
import subprocess

import numpy as np
import pytest

import bench
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _binary(nb):
    b = os.path.join(ROOT, "oracle", "_ref", "seis_ref" if nb == 32 else f"seis_ref_nb{nb}")
    if not os.path.exists(b):
        pytest.skip(f"{b} not built (needs the reference tree at build time)")
    return b


def _reference(wd, vp, rho, d, nb, T, dt, f, src, rec):
    """One shot through the reference binary; returns (seis [nrec][nt], src,
    rec) with the positions as the reference parsed them."""
    nx, nz = vp.shape
    os.makedirs(wd, exist_ok=True)
    np.ascontiguousarray(vp, np.float32).tofile(os.path.join(wd, "vp.bin"))
    np.ascontiguousarray(rho, np.float32).tofile(os.path.join(wd, "rho.bin"))
    with open(os.path.join(wd, "geom.txt"), "w") as fh:
        for gx, gz in rec:
            fh.write(f"{src[0]:.6f},{src[1]:.6f},{gx:.6f},{gz:.6f}\n")
    card = {"Velocity": "vp.bin", "Density": "rho.bin", "NX": nx, "NZ": nz, "DX": d, "DZ": d, "Time": T,
            "FD DT": dt, "DATA DT": dt, "Frequency": f, "Read source receiver flag": 0,
            "if choice=0, Geometry file": "geom.txt", "if choice=1, Shot file": "NA", "Output Directory": "out",
            "Free surface": 0, "Job type New or Restart": "New", "Order of FD Operator": 4}
    with open(os.path.join(wd, "job.json"), "w") as fh:
        fh.write('"Model" : "comment"\n')
        for k, v in card.items():
            fh.write(f'    "{k}" : "{v!r}"\n' if isinstance(v, float) else f'    "{k}" : "{v}"\n')
    os.makedirs(os.path.join(wd, "out"), exist_ok=True)
    r = subprocess.run([_binary(nb), "--no-stability", "job.json"], cwd=wd, capture_output=True, text=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count())))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    g = np.loadtxt(os.path.join(wd, "test_geometry.txt"), dtype=np.float64, ndmin=2)
    src_r = (float(np.float32(g[0, 1])), float(np.float32(g[0, 0])))
    rec_r = np.stack([g[1:, 1], g[1:, 0]], axis=1).astype(np.float32)
    seis = np.fromfile(os.path.join(wd, "out", "job_seismogram.bin"), np.float32).reshape(rec_r.shape[0], -1)
    return seis, src_r, rec_r


def _report(name, got, ref, nt):
    errs = {}
    for q in (1, 2, 3, 4):
        n = max(1, ref.shape[1] * q // 4)
        errs[f"{q}/4"] = O.rel_l2(got[:, :n], ref[:, :n])
    rec = {"config": name, "fd_steps": nt, "rel_l2": errs["4/4"], "rel_l2_by_record_fraction": errs,
           "max_abs_ref": float(np.abs(ref).max())}
    print("PARITY " + json.dumps(rec))
    path = os.environ.get("S2D_PARITY_JSON")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(rec) + "\n")
    return errs["4/4"]


def _ours(models, shots, T, dt, f):
    """models: [(vp, rho, d, nb)]; shots: [(model index, src, rec)] -> traces per shot."""
    from seis2d_b200 import Context, Shot, Wave
    with Context(0) as ctx:
        ms = [ctx.model(vp, rho, d, d, nb) for vp, rho, d, nb in models]
        return ctx.forward([Shot(ms[i], s, r) for i, s, r in shots], Wave(T, dt, dt, f))


def _surface(n, d):
    return np.stack([np.arange(n, dtype=np.float32) * np.float32(d), np.full(n, 2 * d, np.float32)], 1)


def _single(name, tmp_path, vp, rho, d, nb, T, dt, f, src, rec):
    ref, src_r, rec_r = _reference(str(tmp_path / name), vp, rho, d, nb, T, dt, f, src, rec)
    got = _ours([(vp, rho, d, nb)], [(0, src_r, rec_r)], T, dt, f)[0]
    assert got.shape == ref.shape
    err = _report(name, got, ref, bench._ref_fd_nt(T, dt))
    assert err <= TOL, err


def test_c1_two_layer_1000_full_job(tmp_path):
    w = bench.WORKLOADS["c1"]
    vp, rho, src, rec = bench.build_workload(w)
    _single("c1", tmp_path, vp, rho, w["d"], w["nb"], w["T"], w["dt"], w["f"], src[0], rec)


def test_c2_two_layer_5000_first_1000_steps(tmp_path):
    w = bench.WORKLOADS["c2"]
    vp, rho, src, rec = bench.build_workload(w)
    _single("c2", tmp_path, vp, rho, w["d"], w["nb"], 0.5, w["dt"], w["f"], src[0], rec)


def test_c3_salt_full_10000_steps(tmp_path):
    vp, rho = bench.salt_model()
    d = 7.62
    src = (float(np.float32(1600) * np.float32(d)), float(np.float32(2) * np.float32(d)))
    _single("c3", tmp_path, vp, rho, d, 50, 6.0, 0.0006, 20.0, src, _surface(3201, d))


def test_c4_uneven_models_one_batched_call(tmp_path):
    T, dt, f, d, nb = 2.3996, 0.0008, 15.0, 10.0, 50
    models, shots, refs = [], [], []
    for k, (nx, nz) in enumerate([(601, 301), (1201, 601), (2401, 801)]):
        vp, rho = bench.layered_model(nx, nz, 20261203 + 40 + k)
        srcs, rec = bench.surface_shots(nx, d, 16)
        ref, src_r, rec_r = _reference(str(tmp_path / f"c4_{k}"), vp, rho, d, nb, T, dt, f, srcs[8], rec)
        models.append((vp, rho, d, nb))
        shots.append((k, src_r, rec_r))
        refs.append(ref)
    got = _ours(models, shots, T, dt, f)
    for k in range(3):
        assert got[k].shape == refs[k].shape
        err = _report(f"c4_model{k}", got[k], refs[k], bench._ref_fd_nt(T, dt))
        assert err <= TOL, (k, err)


def test_c5_fwi_true_model_forward(tmp_path):
    true, _, rho = bench.fwi_models()
    srcs, rec = bench.surface_shots(1201, 10.0, 32)
    _single("c5", tmp_path, true, rho, 10.0, 50, 3.0, 0.001, 10.0, srcs[16], rec)
