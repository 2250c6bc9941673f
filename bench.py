"""Benchmark of the SeisAcoMod2D forward-modelling hot path on B200.

Workload (default ``c2``): two-layer model on a 5000 x 5000 grid, dx = dz = 5 m,
vp 2000/3500 m/s, rho 1800/2300 kg/m^3 with the interface at 2500 cells,
60-cell sponge (5120 x 5120 padded), 20 Hz Ricker, dt = 0.5 ms, nt = 4000,
64 shots per GPU evenly spaced along the surface (depth 2 cells), each recorded
by 5000 surface receivers; all shots of a GPU advance together (batched).

A bench step advances the whole batch by ``chunk`` FD steps (default 200) of
that job, continuing from the previous step's wavefields, with source
injection and receiver recording exactly as in the full run; the metric is a
rate (padded-cell updates per second), so the full 4000-step job runs at the
same rate.  Inputs (models, shot tables, wavefields) stay in HBM; the state
of 64 shots (54 GB) is far larger than L2, so no L2 flush is needed.

Printed: one JSON line with the metric, the end-to-end rate through the C ABI
from pinned host buffers (``e2e``), the roofline of the step kernel, the
reference CPU path timed on this host (``cpu_baseline``), plain (shot after
shot) vs batched rates, and the SM clocks sampled during the timed region.

``--impl reference`` times the reference's own CPU implementation
(oracle/_ref, SeisAcoMod2D src/src_cpu built unmodified apart from the sponge
width) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per padded-cell update (the library reports them per run
# in stats.alg_bytes): 4 state fields read and written (32 B) + 3 materials
# (12 B) = 44 B; 36 B where both pressure dampings are 1 and the cell carries
# p = px + pz alone.

WORKLOADS = {
    "c2": dict(nx=5000, nz=5000, d=5.0, nb=60, vp=(2000.0, 3500.0), rho=(1800.0, 2300.0), iface=2500,
               f=20.0, dt=0.0005, T=2.0, nshots=64, nrec=5000,
               desc="two-layer 5000x5000 d=5m nb=60, 20 Hz, dt 0.5 ms, nt 4000, 64 shots x 5000 receivers"),
    "c1": dict(nx=1000, nz=1000, d=10.0, nb=40, vp=(1500.0, 3000.0), rho=(1000.0, 2000.0), iface=500,
               f=15.0, dt=0.001, T=2.0, nshots=1, nrec=1000,
               desc="two-layer 1000x1000 d=10m nb=40, 15 Hz, dt 1 ms, nt 2000, 1 shot x 1000 receivers"),
}


# ---------------------------------------------------------------------------
# Seeded synthetic models of the other workload configurations (the
# reference's own model files are not distributed).

def gardner(vp):
    return (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)


def salt_model(seed=20261203 + 3):
    """3201 x 1201, d = 7.62 m: 60 cells of water (1500 m/s), then 1600 -> 4000 m/s
    with a +-5% smoothed Gaussian perturbation, and a 12-vertex salt polygon
    (4500 m/s) in the middle third; Gardner density."""
    from scipy.ndimage import gaussian_filter
    nx, nz = 3201, 1201
    rng = np.random.default_rng(seed)
    z = np.arange(nz, dtype=np.float64)[None, :]
    base = 1600.0 + 2400.0 * (z - 60) / (nz - 1 - 60)
    g = gaussian_filter(rng.standard_normal((nx, nz)), 10.0)
    g /= g.std()
    vp = base * (1.0 + 0.05 * g)
    vp[:, :60] = 1500.0
    cx, cz, R = rng.uniform(nx / 3, 2 * nx / 3), rng.uniform(400, 800), 300.0
    ang = np.sort(rng.uniform(0, 2 * np.pi, 12))
    rad = rng.uniform(0.5, 1.0, 12) * R
    px, pz = cx + rad * np.cos(ang), cz + rad * np.sin(ang)
    X, Z = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(nz, dtype=np.float64), indexing="ij")
    inside = np.zeros((nx, nz), bool)
    for k in range(12):  # even-odd rule
        x1, z1, x2, z2 = px[k], pz[k], px[(k + 1) % 12], pz[(k + 1) % 12]
        cross = ((z1 > Z) != (z2 > Z)) & (X < (x2 - x1) * (Z - z1) / (z2 - z1 + 1e-300) + x1)
        inside ^= cross
    vp[inside & (Z >= 60)] = 4500.0
    vp = vp.astype(np.float32)
    return vp, gardner(vp)


def layered_model(nx, nz, seed):
    """4-8 seeded layers, vp ~ U[1500, 4500], Gardner density."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(4, 9))
    depths = np.sort(rng.uniform(0.1, 0.95, n - 1)) * nz
    vels = rng.uniform(1500.0, 4500.0, n)
    z = np.arange(nz)[None, :].repeat(nx, 0)
    vp = np.full((nx, nz), vels[0], np.float32)
    for k, d in enumerate(depths):
        vp[z >= d] = vels[k + 1]
    return vp, gardner(vp)


def fwi_models(seed=20261203 + 5):
    """1201 x 401, d = 10 m: true = 1500 -> 3500 m/s gradient + two Gaussian
    anomalies of +-300 m/s (sigma 20 cells, seeded centres); start = the
    gradient alone; constant density 2000 kg/m^3 in both."""
    nx, nz = 1201, 401
    rng = np.random.default_rng(seed)
    X, Z = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(nz, dtype=np.float64), indexing="ij")
    start = 1500.0 + 2000.0 * Z / (nz - 1)
    true = start.copy()
    for amp in (300.0, -300.0):
        cx, cz = rng.uniform(200, 1000), rng.uniform(100, 300)
        true += amp * np.exp(-((X - cx) ** 2 + (Z - cz) ** 2) / (2 * 20.0 ** 2))
    rho = np.full((nx, nz), 2000.0, np.float32)
    return true.astype(np.float32), start.astype(np.float32), rho


def build_workload(w, rank=0, world=1):
    nx, nz = w["nx"], w["nz"]
    vp = np.empty((nx, nz), np.float32)
    rho = np.empty((nx, nz), np.float32)
    vp[:, : w["iface"]] = w["vp"][0]
    vp[:, w["iface"]:] = w["vp"][1]
    rho[:, : w["iface"]] = w["rho"][0]
    rho[:, w["iface"]:] = w["rho"][1]
    d = w["d"]
    ntot = w["nshots"] * world
    # shot k of the global list at ix = round((k + 0.5) * nx / ntot), iz = 2
    ks = range(rank * w["nshots"], (rank + 1) * w["nshots"])
    src = [(float(int(round((k + 0.5) * nx / ntot)) * d), 2 * d) for k in ks]
    if w["nshots"] == 1 and world == 1:
        src = [(float(nx // 2) * d, 2 * d)]
    rec = np.stack([np.arange(w["nrec"], dtype=np.float32) * d, np.full(w["nrec"], 2 * d, np.float32)], 1)
    return vp, rho, src, rec


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi's start-up (driver and NVML initialisation, a few hundred
        # ms) can hold up the CUDA calls of this process: let it write its
        # first sample before the timed region begins
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            with open(self.path) as f:
                if f.readline().endswith("\n"):
                    break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(workload, nshots, variant=None):
    """Measured DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum)
    of one step launch over ``nshots`` shots, from the committed ncu summary
    (profiles/traffic.json), scaled from the captured shot count by the
    bytes that grow with the shot count (the state) plus the per-model part
    that does not (the materials), as that file records them."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        t = json.load(open(p)).get(workload)
        if variant is not None and int(t.get("variant", variant)) != int(variant):
            return None  # captured for another step kernel
        b = float(t["per_shot_bytes"]) * nshots + float(t.get("per_model_bytes", 0.0))
        return {"bytes": b, "source": t["source"]}
    except (TypeError, KeyError, ValueError):
        return None


def dram_minimal_bytes(w, nshots):
    """DRAM bytes per padded-cell update if the state crosses HBM once per FD
    step and the materials once per launch for all shots of the model:
    state 32 B per cell (24 B where the cell carries p alone), materials
    12 B / nshots.  Cells carry p alone where both pressure dampings are 1:
    columns and rows [nb-1, n+nb] of the padded grid."""
    nnx, nnz, nb = w["nx"] + 2 * w["nb"], w["nz"] + 2 * w["nb"], w["nb"]
    inner = (nnx - 2 * (nb - 1)) * (nnz - 2 * (nb - 1))
    frac = inner / (nnx * nnz)
    return 24.0 * frac + 32.0 * (1 - frac) + 12.0 / max(1, nshots)


# ---------------------------------------------------------------------------
# Other configurations: single-shot c1/c3, uneven batch c4, gradient c5

def _timed(fn):
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3, out


def surface_shots(nx, d, nshots, nrec=None):
    src = [(float(int(round((k + 0.5) * nx / nshots)) * d), 2 * d) for k in range(nshots)]
    n = nrec or nx
    rec = np.stack([np.arange(n, dtype=np.float32) * d, np.full(n, 2 * d, np.float32)], 1)
    return src, rec


def phase_split(stats, t_forward_s):
    """The gradient call's device time by phase (the library's CUDA events),
    each as a multiple of the forward's time: the forward sweep, the
    recomputes with products, the adjoint steps and the rest (set-up, adjoint
    source, finalisation)."""
    tf = t_forward_s * 1e3
    ph = {"sweep": stats.sweep_ms, "recompute": stats.recompute_ms, "adjoint": stats.adjoint_ms}
    ph["other"] = stats.loop_ms - sum(ph.values())
    return {k: round(v / tf, 3) for k, v in ph.items()}


def gradient_leg(ctx, nshots=32, T=3.0, fd_order=4):
    """FWI gradient on the 1201 x 401 models of fwi_models (nb 50, 10 Hz,
    dt 1 ms, T seconds; 4th- or 8th-order operator): the forward of `nshots`
    shots, then one warm-up gradient and one timed gradient of the same shots,
    timed with CUDA events."""
    import torch
    from seis2d_b200 import Shot, Wave, derive_steps
    true, start, rho = fwi_models()
    wave = Wave(T, 0.001, 0.001, 10.0)
    st = derive_steps(wave)
    src, rec = surface_shots(1201, 10.0, nshots)
    mt = ctx.model(true, rho, 10.0, 10.0, 50, fd_order=fd_order)
    dobs = torch.zeros(nshots * rec.shape[0] * st["real_nt"], dtype=torch.float32, device="cuda")
    ctx.forward([Shot(mt, s_, rec) for s_ in src], wave, out=dobs)
    mt.release()
    ms = ctx.model(start, rho, 10.0, 10.0, 50, fd_order=fd_order)
    shots = [Shot(ms, s_, rec) for s_ in src]
    fbuf = torch.zeros_like(dobs)
    ctx.forward(shots, wave, kt_count=120, out=fbuf)  # autotunes this shape (>= 112 steps) outside the timing
    tf, _ = _timed(lambda: ctx.forward(shots, wave, out=fbuf, sync=False))
    gvp = torch.zeros(1201, 401, dtype=torch.float32, device="cuda")
    grho = torch.zeros_like(gvp)
    # warm-up with the same shot count: an inversion calls the gradient of the
    # same shapes every iteration, its device buffers then come from the pool
    ctx.gradient(shots, wave, dobs, misfit=True, grad_vp=gvp, grad_rho=grho)
    clk = ClockSampler(torch.cuda.current_device())
    clk.start()
    tg, g = _timed(lambda: ctx.gradient(shots, wave, dobs, misfit=True, grad_vp=gvp, grad_rho=grho))
    clocks = clk.stop()
    res = {"workload": f"FWI gradient, 1201x401 (seeded gradient + two +-300 m/s anomalies; start = gradient), "
                       f"rho 2000, nb 50, {nshots} shots x 1201 receivers, nt {st['fd_nt']}, FD order {fd_order}",
           "gradient_s_per_shot": tg / nshots, "forward_s_per_shot": tf / nshots,
           "gradient_over_forward": tg / tf, "misfit": g.misfit,
           "checkpoint_interval": int(g.stats.grad_segment),
           "phases_over_forward": phase_split(g.stats, tf),
           "call_over_loop": round(tg * 1e3 / g.stats.loop_ms, 3),
           "forward_gcells_per_s": ms.padded_cells * nshots * st["fd_nt"] / tf / 1e9,
           "clocks_during_gradient": clocks}
    ms.release()
    return res


def l2_copy_rate():
    """Copy rate of an L2-resident buffer (GB/s, read + write bytes): torch's
    copy of 48 MB into 48 MB (96 MB, inside the 126 MB L2), 20 copies
    captured in a CUDA graph and the graph replayed 10 times, CUDA events —
    the L2 counterpart of the measured HBM copy peak, for the grids whose
    whole state stays in L2 (the graph keeps launch gaps out of the rate)."""
    import torch
    n = 12 * 1024 * 1024
    a = torch.randn(n, device="cuda")
    b = torch.empty_like(a)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(20):
            b.copy_(a)
    g.replay()
    t, _ = _timed(lambda: [g.replay() for _ in range(10)])
    del g
    return 2.0 * 4 * n * 200 / t / 1e9


def extra_legs(device):
    """Rates of the other workload configurations (each a bounded part of its job)."""
    import torch
    from seis2d_b200 import Context, Shot, Wave, derive_steps
    peak, _ = measured_peak()
    out = {}
    with Context(device) as ctx:
        # c1: 1000x1000, nb 40, 15 Hz, dt 1 ms, nt 2000, 1 shot, full job
        w1 = WORKLOADS["c1"]
        vp, rho, src, rec = build_workload(w1)
        m = ctx.model(vp, rho, w1["d"], w1["d"], w1["nb"])
        wave = Wave(w1["T"], w1["dt"], w1["dt"], w1["f"])
        st = derive_steps(wave)
        buf = torch.zeros(rec.shape[0] * st["real_nt"], dtype=torch.float32, device="cuda")
        shots = [Shot(m, src[0], rec)]
        ctx.forward(shots, wave, kt_count=120, out=buf)  # warm-up; autotunes this shape (>= 112 steps)
        t, _ = _timed(lambda: ctx.forward(shots, wave, out=buf, sync=False))
        l1 = ctx.last_stats
        cells = m.padded_cells * st["fd_nt"]
        l2 = l2_copy_rate()
        out["c1"] = {"workload": "1000x1000 two-layer, nb 40, 1 shot, full 2000 steps", "gcells_per_s": cells / t / 1e9,
                     "shots_per_s": 1.0 / t, "job_s": t, "roofline_frac": ctx.last_stats.alg_bytes / t / 1e9 / peak,
                     "l2_copy_gbs": l2, "roofline_frac_l2": ctx.last_stats.alg_bytes / t / 1e9 / l2,
                     "note": "whole job ~37 MB of state: L2-resident; roofline_frac_l2 against the L2 copy rate",
                     "launch": {"variant": l1.variant, "seg_len": l1.seg_len, "task_order": l1.task_order}}
        m.release()
        # c3: salt 3201x1201, d 7.62, nb 50, 20 Hz, dt 0.6 ms, nt 10000, 1 shot; 1000 of the 10000 steps
        vp, rho = salt_model()
        m = ctx.model(vp, rho, 7.62, 7.62, 50)
        wave = Wave(6.0, 0.0006, 0.0006, 20.0)
        st = derive_steps(wave)
        src = (float(1600 * np.float32(7.62)), 2 * 7.62)
        rec = np.stack([np.arange(3201, dtype=np.float32) * np.float32(7.62), np.full(3201, 2 * 7.62, np.float32)], 1)
        buf = torch.zeros(3201 * st["real_nt"], dtype=torch.float32, device="cuda")
        shots = [Shot(m, src, rec)]
        ctx.forward(shots, wave, kt_count=120, out=buf)  # warm-up; autotunes this shape (>= 112 steps)
        t, _ = _timed(lambda: ctx.forward(shots, wave, kt_begin=120, kt_count=1000, out=buf, sync=False))
        cells = m.padded_cells * 1000
        rate = cells / t / 1e9
        frac = ctx.last_stats.alg_bytes / t / 1e9 / peak
        l3 = ctx.last_stats
        out["c3"] = {"workload": "3201x1201 salt (seeded), d 7.62, nb 50, 1 shot, 1000 of 10000 steps",
                     "gcells_per_s": rate, "shots_per_s": rate * 1e9 / (m.padded_cells * st["fd_nt"]),
                     "roofline_frac": frac, "launch": {"variant": l3.variant, "seg_len": l3.seg_len, "task_order": l3.task_order}}
        m.release()
        # c4: 48 shots on three layered models of uneven size, one launch sequence; 300 of 3000 steps
        wave = Wave(2.3996, 0.0008, 0.0008, 15.0)
        st = derive_steps(wave)
        shots, cells_step, total_rec = [], 0, 0
        models = []
        for k, (nx, nz) in enumerate([(601, 301), (1201, 601), (2401, 801)]):
            vp, rho = layered_model(nx, nz, 20261203 + 40 + k)
            mm = ctx.model(vp, rho, 10.0, 10.0, 50)
            models.append(mm)
            src, rec = surface_shots(nx, 10.0, 16)
            shots += [Shot(mm, s_, rec) for s_ in src]
            cells_step += 16 * mm.padded_cells
            total_rec += 16 * rec.shape[0]
        buf = torch.zeros(total_rec * st["real_nt"], dtype=torch.float32, device="cuda")
        ctx.forward(shots, wave, kt_count=120, out=buf)  # warm-up; autotunes this shape (>= 112 steps)
        t, _ = _timed(lambda: ctx.forward(shots, wave, kt_begin=120, kt_count=300, out=buf, sync=False))
        rate = cells_step * 300 / t / 1e9
        frac = ctx.last_stats.alg_bytes / t / 1e9 / peak
        l4 = ctx.last_stats
        ctx.forward(shots, wave, kt_count=60, out=buf, plain=True)  # warm-up of the plain launch sequence
        tp, _ = _timed(lambda: ctx.forward(shots, wave, kt_count=300, out=buf, plain=True, sync=False))
        prate = cells_step * 300 / tp / 1e9
        out["c4"] = {"workload": "48 shots on 601x301 / 1201x601 / 2401x801 layered models (16 each), nb 50, "
                                 "one launch per step for all; 300 of 3000 steps",
                     "gcells_per_s": rate, "shots_per_s": rate * 1e9 / (cells_step / 48 * st["fd_nt"]),
                     "plain_gcells_per_s": prate, "roofline_frac": frac,
                     "launch": {"variant": l4.variant, "seg_len": l4.seg_len, "task_order": l4.task_order}}
        for mm in models:
            mm.release()
        # the 8th-order operator ("Order of FD Operator" : "8") on the 5000x5000
        # two-layer model: 16 of its 64 shots, 200 steps after a warm-up that
        # autotunes the shape (same algorithmic bytes per cell as order 4)
        try:
            w2 = WORKLOADS["c2"]
            vp, rho, src2, rec2 = build_workload(w2)
            m = ctx.model(vp, rho, w2["d"], w2["d"], w2["nb"], fd_order=8)
            wave = Wave(w2["T"], w2["dt"], w2["dt"], w2["f"])
            st = derive_steps(wave)
            shots = [Shot(m, s_, rec2) for s_ in src2[:16]]
            buf = torch.zeros(16 * rec2.shape[0] * st["real_nt"], dtype=torch.float32, device="cuda")
            ctx.forward(shots, wave, kt_count=70, out=buf)  # autotunes the shape (>= 64 steps)
            t, _ = _timed(lambda: ctx.forward(shots, wave, kt_begin=70, kt_count=200, out=buf, sync=False))
            l8 = ctx.last_stats
            rate = 16 * m.padded_cells * 200 / t / 1e9
            out["c2_order8"] = {"workload": "5000x5000 two-layer, nb 60, 8th-order operator, 16 shots x 5000 "
                                            "receivers; 200 of 4000 steps",
                                "gcells_per_s": rate, "roofline_frac": l8.alg_bytes / t / 1e9 / peak,
                                "launch": {"variant": l8.variant, "seg_len": l8.seg_len, "task_order": l8.task_order}}
            m.release()
            del buf
        except Exception as exc:  # a failed extra leg must not cost the main line
            out["c2_order8"] = {"error": str(exc)}
        # c5: FWI gradient, 32 shots, 1201x401, nb 50, 10 Hz, dt 1 ms, nt 3000
        # checkpoint every 100 steps, as the configuration states
        ctx.set_option("grad_segment", 100)
        out["c5_gradient"] = gradient_leg(ctx, 32, 3.0)
        # the same with the 8th-order operator (its adjoint is the two-pass
        # cell-parallel form); a failed extra leg must not cost the main line
        try:
            out["c5_gradient_order8"] = gradient_leg(ctx, 32, 3.0, fd_order=8)
        except Exception as exc:
            out["c5_gradient_order8"] = {"error": str(exc)}
        ctx.set_option("grad_segment", 0)
    return out


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref, the reference's own src/src_cpu)

def _ref_fd_nt(T, dt):
    """FD steps of a run as the reference derives them: ceil of the float32
    quotient Time / FD DT (src/src_cpu/cpumodelling.cpp:174)."""
    return int(math.ceil(float(np.float32(T) / np.float32(dt))))


def _write_ref_job(wd, w, vp, rho, src, T):
    """The reference's input files for one shot of workload ``w``: raw float32
    [nx][nz] models, a one-line shot file (split spread) and a job card
    (src/src_cpu/json_parser.cpp:122-300, create_geometry.cpp:72-143)."""
    np.ascontiguousarray(vp, np.float32).tofile(os.path.join(wd, "vp.bin"))
    np.ascontiguousarray(rho, np.float32).tofile(os.path.join(wd, "rho.bin"))
    with open(os.path.join(wd, "shots.txt"), "w") as f:
        f.write(f"{src[0]:.6f},{src[1]:.6f},{int(w['nrec'])},0,{w['d']:.6f},1\n")
    card = {"Velocity": "vp.bin", "Density": "rho.bin", "NX": w["nx"], "NZ": w["nz"], "DX": w["d"],
            "DZ": w["d"], "Time": T, "FD DT": w["dt"], "DATA DT": w["dt"], "Frequency": w["f"],
            "Read source receiver flag": 1, "if choice=0, Geometry file": "NA",
            "if choice=1, Shot file": "shots.txt", "Output Directory": "out", "Free surface": 0,
            "Job type New or Restart": "New", "Order of FD Operator": 4}
    with open(os.path.join(wd, "job.json"), "w") as f:
        f.write('"Model" : "comment"\n')
        for k, v in card.items():
            f.write(f'    "{k}" : "{v!r}"\n' if isinstance(v, float) else f'    "{k}" : "{v}"\n')


def ref_cpu_rate(w, nsteps_pair=(4, 84), threads=None, tmpdir=None):
    """Gcell/s of the reference CPU time loop on one shot of workload ``w``:
    two runs of nsteps_pair FD steps, rate from the difference (set-up cancels).
    Runs only the reference binary (oracle/_ref); imports nothing of the
    modelling package."""
    nb = w["nb"]
    binary = os.path.join(ROOT, "oracle", "_ref", "seis_ref" if nb == 32 else f"seis_ref_nb{nb}")
    if not os.path.exists(binary):
        return None, f"{binary} not built"
    vp, rho, src, rec = build_workload(dict(w, nshots=1), 0, 1)
    times = []
    env = dict(os.environ)
    threads = threads or os.cpu_count()
    env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory(dir=tmpdir) as wd:
        os.makedirs(os.path.join(wd, "out"))
        for n in nsteps_pair:
            T = n * w["dt"]
            _write_ref_job(wd, w, vp, rho, src[0], T)
            r = subprocess.run([binary, "--no-stability", "--time", "job.json"], cwd=wd, env=env,
                               capture_output=True, text=True)
            if r.returncode != 0:
                return None, f"reference exited {r.returncode}"
            t = [float(l.split()[1]) for l in r.stdout.splitlines() if l.startswith("ORACLE_TIME")]
            times.append((t[0], _ref_fd_nt(T, w["dt"])))
    (t0, n0), (t1, n1) = times
    cells = (w["nx"] + 2 * nb) * (w["nz"] + 2 * nb)
    rate = cells * (n1 - n0) / max(t1 - t0, 1e-9) / 1e9
    sample = (f"1 shot of the workload, {n0} and {n1} FD steps ({t0:.2f} s, {t1:.2f} s wall incl. set-up); "
              f"rate from the difference")
    return {"value": rate, "unit": "Gcell/s", "cores": threads, "kind": "reference", "sample": sample}, None


def run_reference_arm(args, w, world, rank):
    if rank != 0:
        return 0
    vals = []
    info = None
    # Each step is one bounded sample (two short runs of one shot); warm-up
    # samples are shorter still.
    for _ in range(min(args.warmup, 1)):
        ref_cpu_rate(w, (2, 4))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        info, err = ref_cpu_rate(w)
        if info is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return 0
        vals.append(info["value"])
    wall = time.perf_counter() - t0
    v = statistics.median(vals)
    info["value"] = v
    line = {
        "impl": "reference", "metric": "padded-grid cell-updates per second, batched forward modelling",
        "value": v, "unit": "Gcell/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["desc"], "sample": info["sample"]},
        "cpu_baseline": info, "e2e": {"value": v, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--chunk", type=int, default=200, help="FD steps per bench step")
    ap.add_argument("--shots", type=int, default=0, help="override shots per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the c1/c3/c4/c5 legs")
    ap.add_argument("--variant", type=int, default=-1,
                    help="force a step-kernel variant (s2d_set_option 'variant'); default: autotuned")
    ap.add_argument("--task-order", type=int, default=-1, choices=[-1, 0, 1],
                    help="force the task order (s2d_set_option 'task_order'); default: autotuned")
    ap.add_argument("--leg", default="main", choices=["main", "gradient"],
                    help="gradient: only the FWI gradient leg (--shots shots, --grad-time seconds)")
    ap.add_argument("--grad-time", type=float, default=3.0, help="record length of the gradient leg (s)")
    ap.add_argument("--grad-segment", type=int, default=0, help="checkpoint interval of the gradient leg (0: auto)")
    ap.add_argument("--adjoint-blocks", type=int, default=0,
                    help="gradient leg: s2d_set_option 'adjoint_blocks' (0: library default)")
    ap.add_argument("--products-variant", type=int, default=0,
                    help="gradient leg: s2d_set_option 'products_variant' (0: library default)")
    ap.add_argument("--fd-order", type=int, default=4, choices=[4, 8],
                    help="FD operator of the main leg: 4 (the reference's) or 8 (Order of FD Operator = 8)")
    args = ap.parse_args()
    if args.leg == "gradient":
        import torch
        from seis2d_b200 import Context
        with Context(0) as ctx:
            ctx.set_option("grad_segment", args.grad_segment)
            if args.variant >= 0:
                ctx.set_option("variant", args.variant)
            if args.task_order >= 0:
                ctx.set_option("task_order", args.task_order)
            if args.products_variant:
                ctx.set_option("products_variant", args.products_variant)
            if args.adjoint_blocks:
                ctx.set_option("adjoint_blocks", args.adjoint_blocks)
            leg = "c5_gradient" if args.fd_order == 4 else "c5_gradient_order8"
            print(json.dumps({"leg": leg, **gradient_leg(ctx, args.shots or 32, args.grad_time, args.fd_order)}))
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = dict(WORKLOADS[args.workload])
    if args.shots:
        w["nshots"] = args.shots
    if args.impl == "reference":
        return run_reference_arm(args, w, world, rank)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from seis2d_b200 import Context, Shot, Wave, derive_steps

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    wave = Wave(w["T"], w["dt"], w["dt"], w["f"])
    steps = derive_steps(wave)
    fd_nt = steps["fd_nt"]
    chunk = max(1, min(args.chunk, fd_nt // max(1, args.warmup + args.steps)))
    vp, rho, src, rec = build_workload(w, rank, world)
    nshots = len(src)
    cells_shot = (w["nx"] + 2 * w["nb"]) * (w["nz"] + 2 * w["nb"])
    cells_step = cells_shot * nshots  # per FD step, this rank

    ctx = Context(local)
    if args.variant >= 0:
        ctx.set_option("variant", args.variant)
    if args.task_order >= 0:
        ctx.set_option("task_order", args.task_order)
    m = ctx.model(vp, rho, w["d"], w["d"], w["nb"], fd_order=args.fd_order)
    shots = [Shot(m, s, rec) for s in src]
    nrec_tot = nshots * rec.shape[0]
    seis_dev = torch.zeros(nrec_tot * steps["real_nt"], dtype=torch.float32, device="cuda")

    # ---- batched, device-resident (value) ----
    kt = 0
    launches = 0
    tune = None
    for _ in range(args.warmup):
        ctx.forward(shots, wave, kt_begin=kt, kt_count=chunk, out=seis_dev)
        kt += chunk
        st = ctx.last_stats
        if tune is None or st.autotuned:
            tune = {"variant": st.variant, "block": st.block, "stages": st.stages, "seg_len": st.seg_len,
                    "task_order": st.task_order, "autotuned_in_warmup": bool(st.autotuned)}
    barrier()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loop_ms = alg_bytes = 0.0
    fd_launches = 0
    variants = set()
    ev0.record()
    for _ in range(args.steps):
        ctx.forward(shots, wave, kt_begin=kt, kt_count=chunk, out=seis_dev, sync=False)
        st = ctx.last_stats
        launches += st.kernel_launches
        # the library's own CUDA events around its step launches, on the
        # stream it launches them on, and the algorithmic bytes of those steps
        loop_ms += st.loop_ms
        alg_bytes += st.alg_bytes
        fd_launches += -(-chunk // (2 if st.variant == 5 else 1))
        variants.add(int(st.variant))
        kt += chunk
    ev1.record()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    t_max = torch.tensor([ms], device="cuda")
    if dist is not None:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms = float(t_max.item())
    total_cells = cells_step * chunk * args.steps * world
    value = total_cells / (ms * 1e-3) / 1e9
    ms_per_step = ms / args.steps

    # roofline of the step kernel over exactly the timed calls: algorithmic
    # bytes of the launches / their device time (library events on its stream)
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (loop_ms * 1e-3) / 1e9
    tr = traffic_per_launch(args.workload, nshots, next(iter(variants)) if len(variants) == 1 else None)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr["bytes"] if tr else None, "traffic_source": tr["source"] if tr else None,
            "peak_source": peak_kind, "bytes_per_launch": alg_bytes / max(1, fd_launches),
            "bytes_per_cell_update": alg_bytes / (cells_step * chunk * args.steps),
            "dram_minimal_bytes_per_cell_update": dram_minimal_bytes(w, nshots),
            "launch_ms": loop_ms / max(1, fd_launches), "launches": fd_launches,
            "fd_steps_per_launch": 2 if variants == {5} else 1,
            "timed_region": f"the {args.steps} timed calls ({fd_launches} step launches)"}
    if variants == {5}:
        # the two-step kernel moves the state once per two steps: the fraction
        # of the peak a one-step kernel would need for the same rate
        one = roof["bytes_per_cell_update"] * 2
        roof["one_step_equivalent"] = {"bytes_per_cell_update": one,
                                       "frac": total_cells * one / (ms * 1e-3) / 1e9 / world / peak}

    # ---- end to end through the C ABI from pinned host memory ----
    e2e = None
    if not args.no_e2e:
        vp_h = torch.from_numpy(vp).pin_memory()
        rho_h = torch.from_numpy(rho).pin_memory()
        out_h = torch.zeros(nrec_tot * steps["real_nt"], dtype=torch.float32).pin_memory()
        short = Wave(chunk * w["dt"], w["dt"], w["dt"], w["f"])
        real_short = derive_steps(short)["real_nt"]
        out_h = out_h[: nrec_tot * real_short]
        n_e2e = max(1, min(args.steps, 3))

        loop_s = []

        def one():
            mm = ctx.model(vp_h.numpy(), rho_h.numpy(), w["d"], w["d"], w["nb"], fd_order=args.fd_order)
            ctx.forward([Shot(mm, s, rec) for s in src], short, out=out_h.numpy())
            loop_s.append(ctx.last_stats.loop_ms * 1e-3)
            mm.release()

        one()
        barrier()
        eclk = ClockSampler(torch.cuda.current_device())
        eclk.start()
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            one()
        barrier()
        et = torch.tensor([time.perf_counter() - t0], device="cuda")
        eclocks = eclk.stop()
        if dist is not None:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        ecells = cells_step * derive_steps(short)["fd_nt"] * n_e2e * world
        e2e = {"value": ecells / float(et.item()) / 1e9, "unit": "Gcell/s",
               "h2d_bytes_per_step": int(vp.nbytes + rho.nbytes),
               "d2h_bytes_per_step": int(nrec_tot * real_short * 4),
               "sample": f"{n_e2e} calls: model upload + {nshots} shots x {derive_steps(short)['fd_nt']} FD steps "
                         f"+ seismogram download, pinned host buffers", "clocks": eclocks,
               "wall_s_per_call": float(et.item()) / n_e2e, "loop_s_per_call": sum(loop_s[1:]) / n_e2e}

    # ---- plain: the same shots one after another ----
    plain = None
    if not args.no_plain and nshots > 1:
        pch = max(1, chunk // 4)
        ctx.forward(shots, wave, kt_begin=0, kt_count=pch, out=seis_dev, plain=True)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.forward(shots, wave, kt_begin=pch, kt_count=pch, out=seis_dev, plain=True, sync=False)
        e1.record()
        barrier()
        pms = e0.elapsed_time(e1)
        prate = cells_step * pch / (pms * 1e-3) / 1e9
        plain = {"value": prate * world, "unit": "Gcell/s", "speedup_batched_vs_plain": value / (prate * world),
                 "sample": f"{nshots} shots x {pch} FD steps, shot after shot"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, err = ref_cpu_rate(w)
        if cpu is None:
            cpu = {"unavailable": err}
        else:
            # the 1000 x 1000 case on one thread and on all host threads
            # (bounded samples: 4 and 204 FD steps of one shot)
            c1 = WORKLOADS["c1"]
            one, _ = ref_cpu_rate(c1, (4, 204), threads=1)
            allc, _ = ref_cpu_rate(c1, (4, 204))
            cpu["c1_reference"] = {"one_thread": one, "all_threads": allc}

    ctx.close()
    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        torch.cuda.empty_cache()
        extras = extra_legs(local)
    if rank == 0:
        line = {
            "metric": "padded-grid cell-updates per second, batched forward modelling",
            "value": value, "unit": "Gcell/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["desc"] + ("" if args.fd_order == 4 else ", 8th-order operator"),
                       "shots_per_gpu": nshots, "fd_steps_per_bench_step": chunk,
                       "padded_grid": [w["nx"] + 2 * w["nb"], w["nz"] + 2 * w["nb"]],
                       "l2": "inputs larger than L2 (wavefield state %.1f GB per GPU)" % (cells_step * 32 / 1e9),
                       "parallelism": f"shots sharded over {world} GPU(s), no collective",
                       "launch": tune},
            "shots_per_s": value * 1e9 / (cells_shot * fd_nt),
            "physical_gcells_per_s": value * (w["nx"] * w["nz"]) / cells_shot,
            "plain": plain, "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": launches, "other_configs": extras,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
