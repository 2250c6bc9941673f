"""The reference's file-level job handling, through the C ABI host driver
(``seis2d_b200/csrc/s2d_driver.cpp``):

    card = read_jobcard("input/job.json")        # json_parser.cpp:13-300
    geom = read_geometry(card)                   # create_geometry.cpp / read_receiver.cpp
    run_jobcard("input/job.json", naming="gpu")  # Modelling_master + modelling_module

Errors raise ``Seis2dError`` whose message names the reference's abort code.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Tuple

import numpy as np

from . import _lib as L


def _err():
    return C.create_string_buffer(1024)


def read_jobcard(path: str) -> L.JobCard:
    card = L.JobCard()
    eb = _err()
    rc = L.lib().s2d_jobcard_read(path.encode(), C.byref(card), eb, 1024)
    if rc:
        raise L.Seis2dError(rc, eb.value.decode())
    return card


def read_geometry(card: L.JobCard) -> List[Tuple[Tuple[float, float], np.ndarray]]:
    """``[((sx, sz), rec[nrec][2]), ...]`` in metres, float32 as the reference holds them."""
    g = L.Geometry()
    eb = _err()
    rc = L.lib().s2d_geometry_read(C.byref(card), C.byref(g), eb, 1024)
    if rc:
        raise L.Seis2dError(rc, eb.value.decode())
    try:
        out = []
        for s in range(g.nsrc):
            n = g.nrec[s]
            rec = np.ctypeslib.as_array(C.cast(g.rec[s], C.POINTER(C.c_float)), shape=(n * 2,)).copy().reshape(n, 2)
            out.append(((g.src[s].x, g.src[s].z), rec))
        return out
    finally:
        L.lib().s2d_geometry_free(C.byref(g))


def check_stability(card: L.JobCard, vmin: float, vmax: float) -> None:
    eb = _err()
    rc = L.lib().s2d_check_stability(C.byref(card), vmin, vmax, eb, 1024)
    if rc:
        raise L.Seis2dError(rc, eb.value.decode())


def run_jobcard(path: str, device: int = 0, nb: int = 32, naming: str = "cpu", check_stability: bool = True,
                verbose: bool = False, rank: int = 0, nranks: int = 1) -> None:
    """The whole job (rank 0 of 1), or rank ``rank``'s block of shots of an
    ``nranks``-process job (see seis2d_b200.sharding.run_jobcard_distributed)."""
    eb = _err()
    rc = L.lib().s2d_run_jobcard_rank(path.encode(), int(device), int(nb), 1 if naming == "gpu" else 0,
                                      1 if check_stability else 0, 1 if verbose else 0, int(rank), int(nranks),
                                      eb, 1024)
    if rc:
        raise L.Seis2dError(rc, eb.value.decode())
