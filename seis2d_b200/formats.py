"""File formats of SeisAcoMod2D kept byte-compatible by this package.

* Job card: one ``"Key" : "Value"`` pair per line; lines containing
  ``comment``/``Comment`` are skipped (src/src_cpu/json_parser.cpp:56-77).
* Shot file: ``sx,sz,nrec,nearoff,spacing,type`` per line, metres, type 1
  split, 2 end-on-left, 3 end-on-right (src/src_cpu/create_geometry.cpp:72-143).
* Explicit geometry file: ``sx,sz,gx,gz`` per line, grouped per shot and
  sorted by sx (src/src_cpu/read_receiver.cpp:162-306).
* Model: raw float32, x-major ``[nx][nz]`` with z fastest
  (src/src_cpu/model.cpp:12-44).
* Seismogram: raw float32 ``[nrec][nt]``, sample fastest
  (src/src_cpu/cpumodelling.cpp:367-374).

These helpers write the inputs a user of the reference would write and read
the outputs it produces.  The parsing used by the modelling path itself is the
C++ host driver in ``seis2d_b200/csrc/s2d_driver.cpp``.
"""
from __future__ import annotations

import os
from typing import Dict, Iterable, Sequence, Tuple

import numpy as np

# Key names exactly as src/src_cpu/json_parser.cpp:128-265 looks them up.
JOBCARD_KEYS = (
    "Velocity", "Density", "NX", "NZ", "DX", "DZ", "Time", "FD DT", "DATA DT",
    "Frequency", "Read source receiver flag", "if choice=0, Geometry file",
    "if choice=1, Shot file", "Output Directory", "Free surface",
    "Job type New or Restart", "Order of FD Operator",
)


def write_model(path: str, arr: np.ndarray) -> None:
    """Write a ``[nx][nz]`` model as raw little-endian float32."""
    a = np.ascontiguousarray(arr, dtype=np.float32)
    if a.ndim != 2:
        raise ValueError("model must be 2-D [nx][nz]")
    a.tofile(path)


def read_model(path: str, nx: int, nz: int) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float32)
    if a.size != nx * nz:
        raise ValueError(f"{path}: expected {nx*nz} float32 values, found {a.size}")
    return a.reshape(nx, nz)


def read_seismogram(path: str, nrec: int) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float32)
    if a.size % nrec:
        raise ValueError(f"{path}: {a.size} samples is not a multiple of nrec={nrec}")
    return a.reshape(nrec, a.size // nrec)


def _fmt(v) -> str:
    if isinstance(v, float):
        return repr(v)
    return str(v)


def write_jobcard(path: str, params: Dict[str, object]) -> None:
    """Write a job card in the reference's line format.

    ``params`` maps the reference key names (``JOBCARD_KEYS``) to values;
    section headers are written as comment lines the way the shipped cards
    (input/*.json) lay them out.
    """
    lines = ['"Model" : "comment"']
    for k in ("Velocity", "Density", "NX", "NZ", "DX", "DZ", "Time", "FD DT",
              "DATA DT", "Frequency", "Read source receiver flag",
              "if choice=0, Geometry file", "if choice=1, Shot file",
              "Output Directory", "Free surface", "Job type New or Restart",
              "Order of FD Operator"):
        if k in params:
            lines.append(f'    "{k}" : "{_fmt(params[k])}"')
    for k, v in params.items():
        if k not in JOBCARD_KEYS:
            lines.append(f'    "{k}" : "{_fmt(v)}"')
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_shotfile(path: str, shots: Iterable[Tuple[float, float, int, float, float, int]]) -> None:
    """Rows ``(sx, sz, nrec, nearoff, spacing, type)`` in metres."""
    with open(path, "w") as f:
        for sx, sz, nrec, near, sp, gt in shots:
            f.write(f"{sx:.6f},{sz:.6f},{int(nrec)},{near:g},{sp:.6f},{int(gt)}\n")


def write_geometry(path: str, shots: Sequence[Tuple[Tuple[float, float], Sequence[Tuple[float, float]]]]) -> None:
    """Explicit geometry: ``[((sx, sz), [(gx, gz), ...]), ...]`` in metres."""
    with open(path, "w") as f:
        for (sx, sz), recs in shots:
            for gx, gz in recs:
                f.write(f"{sx:.6f},{sz:.6f},{gx:.6f},{gz:.6f}\n")


def jobname_from_card(card_path: str) -> str:
    """Output-name prefix: card basename without extension, plus ``_``
    (src/src_cpu/json_parser.cpp:13-37)."""
    base = os.path.basename(card_path)
    stem = base.rsplit(".", 1)[0] if "." in base else base
    return stem + "_"
