"""ctypes access to the C restatement in ``oracle/s2d_oracle.c``.

TEST INFRASTRUCTURE: imported only by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s cpu_baseline leg, as the checker.  The product path never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN_DIR = os.path.join(HERE, "_ref")

F64 = 64
F32 = 32


class _Params(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nb", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("rec_len", C.c_float),
                ("fd_dt", C.c_float), ("real_dt", C.c_float), ("fm", C.c_float),
                ("free_surface", C.c_int), ("fd_order", C.c_int)]


class _Derived(C.Structure):
    _fields_ = [("nnx", C.c_int), ("nnz", C.c_int), ("fd_nt", C.c_int),
                ("real_nt", C.c_int), ("dt_factor", C.c_int), ("nts", C.c_int),
                ("dtdx", C.c_double), ("dtdz", C.c_double)]


_lib = None


def build() -> str:
    """Compile ``liboracle.so`` with the oracle Makefile (gcc, no GPU)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "s2d_oracle.c")
        if (not os.path.exists(LIB_PATH)
                or os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_derive.argtypes = [C.POINTER(_Params), C.POINTER(_Derived)]
        L.orc_ricker.argtypes = [C.POINTER(_Params), C.POINTER(_Derived), C.POINTER(C.c_double)]
        L.orc_cell.argtypes = [C.POINTER(_Params), C.c_float, C.c_float]
        L.orc_cell.restype = C.c_int
        L.orc_forward.argtypes = [
            C.POINTER(_Params), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
            C.c_float, C.c_float, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
            C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double)]
        L.orc_forward.restype = C.c_int
        dp = C.POINTER(C.c_double)
        L.orc_gradient.argtypes = [
            C.POINTER(_Params), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float, C.c_float, C.c_int,
            C.POINTER(C.c_float), C.POINTER(C.c_float), dp, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp]
        L.orc_gradient.restype = C.c_int
        L.orc_gradient_seg.argtypes = L.orc_gradient.argtypes + [C.c_int]
        L.orc_gradient_seg.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = None
        _lib = L
    return _lib


@dataclass
class Params:
    nx: int
    nz: int
    nb: int
    dx: float
    dz: float
    rec_len: float
    fd_dt: float
    real_dt: float
    fm: float
    free_surface: int = 0  # 1: pressure-release surface at the first model row
    fd_order: int = 4      # 4: the reference's operator; 8: the 8th-order operator

    def c(self) -> _Params:
        return _Params(self.nx, self.nz, self.nb, self.dx, self.dz, self.rec_len,
                       self.fd_dt, self.real_dt, self.fm, int(self.free_surface), int(self.fd_order))


def derive(p: Params) -> dict:
    d = _Derived()
    lib().orc_derive(C.byref(p.c()), C.byref(d))
    return {k: getattr(d, k) for k, _ in _Derived._fields_}


def ricker(p: Params) -> np.ndarray:
    d = _Derived()
    cp = p.c()
    lib().orc_derive(C.byref(cp), C.byref(d))
    w = np.zeros(d.nts, np.float64)
    lib().orc_ricker(C.byref(cp), C.byref(d), w.ctypes.data_as(C.POINTER(C.c_double)))
    return w


def cell(p: Params, x: float, z: float) -> int:
    return lib().orc_cell(C.byref(p.c()), x, z)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def forward(p: Params, vp: np.ndarray, rho: np.ndarray, src: Sequence[float],
            rec_x: Sequence[float], rec_z: Sequence[float], precision: int = F64,
            wavelet: Optional[np.ndarray] = None, kt_stop: int = 0,
            want_state: bool = False):
    """One shot on the CPU restatement.  Returns ``seis[nrec][real_nt]`` and,
    with ``want_state``, ``(px, pz, vx, vz, p)`` as ``[nnx][nnz]`` float64."""
    vp = np.ascontiguousarray(vp, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    assert vp.shape == (p.nx, p.nz) and rho.shape == (p.nx, p.nz)
    gx = np.ascontiguousarray(rec_x, np.float32)
    gz = np.ascontiguousarray(rec_z, np.float32)
    d = derive(p)
    seis = np.zeros((gx.size, d["real_nt"]), np.float32)
    state = np.zeros((5, d["nnx"], d["nnz"]), np.float64) if want_state else None
    wp = None
    nw = 0
    if wavelet is not None:
        wavelet = np.ascontiguousarray(wavelet, np.float64)
        wp = wavelet.ctypes.data_as(C.POINTER(C.c_double))
        nw = wavelet.size
    rc = lib().orc_forward(C.byref(p.c()), precision, _fp(vp), _fp(rho),
                           float(src[0]), float(src[1]), gx.size, _fp(gx), _fp(gz),
                           wp, nw, int(kt_stop), _fp(seis),
                           state.ctypes.data_as(C.POINTER(C.c_double)) if want_state else None)
    if rc != 0:
        raise ValueError(f"orc_forward failed with status {rc}")
    if want_state:
        return seis, tuple(state[i] for i in range(5))
    return seis


def set_threads(n: int) -> None:
    """Threads of the FP64 gradient's loops (same bits for every count)."""
    lib().orc_set_threads(int(n))


def gradient(p: Params, vp: np.ndarray, rho: np.ndarray, src, rec_x, rec_z, adj: Optional[np.ndarray],
             wavelet: Optional[np.ndarray] = None, segment: int = 0):
    """FP64 discrete adjoint of the FP64 forward.  Returns a dict with
    grad_vp, grad_rho ([nx][nz]), grad_kappa, grad_bx, grad_bz ([nnx][nnz]),
    src_adj ([fd_nt]) and seis64 ([nrec][real_nt]).  ``segment``: checkpoint
    interval in FD steps (0: every step's products kept); ``adj=None`` runs
    the forward alone (seis64; the gradients are zero)."""
    vp = np.ascontiguousarray(vp, np.float32)
    rho = np.ascontiguousarray(rho, np.float32)
    gx = np.ascontiguousarray(rec_x, np.float32)
    gz = np.ascontiguousarray(rec_z, np.float32)
    d = derive(p)
    nnx, nnz, nt = d["nnx"], d["nnz"], d["fd_nt"]
    out = {"grad_vp": np.zeros((p.nx, p.nz)), "grad_rho": np.zeros((p.nx, p.nz)),
           "grad_kappa": np.zeros((nnx, nnz)), "grad_bx": np.zeros((nnx, nnz)), "grad_bz": np.zeros((nnx, nnz)),
           "src_adj": np.zeros(nt), "seis64": np.zeros((gx.size, d["real_nt"]))}
    dpp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    wp, nw = None, 0
    if wavelet is not None:
        wavelet = np.ascontiguousarray(wavelet, np.float64)
        wp, nw = dpp(wavelet), wavelet.size
    a = None
    if adj is not None:
        a = np.ascontiguousarray(adj, np.float64)
        assert a.shape == (gx.size, d["real_nt"])
    rc = lib().orc_gradient_seg(C.byref(p.c()), _fp(vp), _fp(rho), float(src[0]), float(src[1]), gx.size,
                                _fp(gx), _fp(gz), wp, nw, dpp(a) if a is not None else None,
                                *(dpp(out[k]) for k in ("grad_vp", "grad_rho", "grad_kappa", "grad_bx", "grad_bz",
                                                        "src_adj", "seis64")), int(segment))
    if rc != 0:
        raise ValueError(f"orc_gradient failed with status {rc}")
    return out


def ref_binary(nb: int = 32) -> str:
    """Path of the reference CPU binary built by ``make -C oracle ref [NB=nb]``."""
    name = "seis_ref" if nb == 32 else f"seis_ref_nb{nb}"
    return os.path.join(REF_BIN_DIR, name)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
