"""Build libseis2d.so in-tree with nvcc for sm_100a.

``python -m seis2d_b200.build`` (or ``__graft_entry__.build()``) compiles every
source of ``seis2d_b200/csrc`` and links ``seis2d_b200/libseis2d.so`` (CUDA
runtime linked statically, so the library carries no dependency on the
toolkit's shared runtime).  nvcc cross-compiles; no GPU is needed.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libseis2d.so")
CLI_SRC = os.path.join(HERE, "cli", "seis2d_run.cpp")
CLI = os.path.join(HERE, "bin", "seis2d_run")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # The plain system compiler; an inherited CXX may be a wrapper.
    return shutil.which("g++") or "g++"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(CLI):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h")) + [CLI_SRC]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-ccbin", _host_cxx(), "-I", os.path.join(ROOT, "include")]
    if os.environ.get("S2D_DEVICE_CHECKS") == "1":
        # debug build: per-task range checks in the step kernels (see s2d_device.cuh)
        common += ["-DS2D_DEVICE_CHECKS"]
    objs = []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        cmd = [nvcc] + ARCH + common + ["-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "cu"] if False else []
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        objs.append(obj)
    cmd = [nvcc] + ARCH + ["-shared", "-ccbin", _host_cxx(), "-o", LIB + ".tmp"] + objs + ["-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    # command-line driver, linked against the library by rpath
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cmd = [_host_cxx(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), CLI_SRC, "-o", CLI,
           "-L", HERE, "-lseis2d", "-Wl,-rpath,$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"seis2d_run link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
