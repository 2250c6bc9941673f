"""bench.py's reference arm under torchrun with two ranks on the CPU: rank 0
times the reference CPU path and prints one JSON line, the other rank exits 0
without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_two_ranks():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "seis_ref_nb60")):
        pytest.skip("reference binary for the bench workload (nb 60) not built")
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "Gcell/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"


def test_reference_arm_loads_no_product_code():
    """The reference arm times the reference binary alone: after one sample
    no module of the modelling package (which would map libseis2d.so) is
    imported."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "seis_ref_nb40")):
        pytest.skip("reference binary for the 1000 x 1000 workload (nb 40) not built")
    code = ("import sys, bench; info, err = bench.ref_cpu_rate(bench.WORKLOADS['c1'], (2, 6), threads=2); "
            "assert info and info['value'] > 0, err; "
            "print(sorted(m for m in sys.modules if m.startswith('seis2d_b200')))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "[]"


def test_roofline_traffic_and_minimal_bytes():
    """The measured-traffic record scales to a launch's shot count, and the
    DRAM-minimal bytes per cell-update lie between the merged-cell 24 B and
    the split-cell 32 B plus the shots' share of the materials."""
    sys.path.insert(0, ROOT)
    import bench
    t2, t64 = bench.traffic_per_launch("c2", 2), bench.traffic_per_launch("c2", 64)
    assert t2 and t64 and t64["bytes"] > 30 * t2["bytes"] / 2 * 0.9
    assert abs(t2["bytes"] - 1.622e9) < 0.01e9  # the measured 2-shot launch
    # the record holds one step kernel's capture: none for another kernel
    assert bench.traffic_per_launch("c2", 64, 16) == t64
    assert bench.traffic_per_launch("c2", 64, 5) is None
    for n in (1, 64):
        b = bench.dram_minimal_bytes(bench.WORKLOADS["c2"], n)
        assert 24.0 + 12.0 / n <= b <= 32.0 + 12.0 / n
