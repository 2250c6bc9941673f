"""ctypes binding of libseis2d (include/seis2d.h).

Loading fails loudly when the in-tree library is missing: there is no CPU
fallback for the modelling path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libseis2d.so")

S2D_OK = 0
S2D_ERR_ARG = -1
S2D_ERR_CUDA = -2
S2D_ERR_NOMEM = -3
S2D_ERR_GEOM = -4
S2D_ERR_STATE = -5
S2D_ERR_IO = -6
S2D_ERR_JOBCARD = -7
S2D_ERR_STABILITY = -8
S2D_ERR_TIMEOUT = -9
S2D_ERR_NODEV = -10

ABI_VERSION = 3  # S2D_ABI_VERSION of include/seis2d.h

S2D_SEIS_DEVICE = 0x1
S2D_PLAIN = 0x2
S2D_NO_GRAPH = 0x4
S2D_SYNC = 0x8
S2D_MODEL_DEVICE = 0x1
S2D_MODEL_FREE_SURFACE = 0x2
S2D_MODEL_ORDER8 = 0x4
S2D_GRAD_MISFIT = 0x10
S2D_GRAD_DEVICE = 0x20
S2D_STATIC_MODEL_DEVICE = 0x100
S2D_STATIC_SEIS_DEVICE = 0x200


class Coord(C.Structure):
    _fields_ = [("x", C.c_float), ("z", C.c_float)]


class Wave(C.Structure):
    _fields_ = [("rec_len", C.c_float), ("fd_dt", C.c_float), ("real_dt", C.c_float), ("dom_freq", C.c_float)]


class Shot(C.Structure):
    _fields_ = [("model_id", C.c_int), ("src", Coord), ("nrec", C.c_int), ("rec", C.POINTER(Coord))]


class Steps(C.Structure):
    _fields_ = [("fd_nt", C.c_int), ("real_nt", C.c_int), ("dt_factor", C.c_int), ("nts", C.c_int)]


class JobCard(C.Structure):
    """s2d_jobcard: the fields the reference fills from a job card."""
    _fields_ = [("velfile", C.c_char * 224), ("densfile", C.c_char * 224), ("nx", C.c_int), ("nz", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("wave", Wave), ("geomflag", C.c_int), ("frsf", C.c_int),
                ("fdop", C.c_int), ("jbtype", C.c_char * 8), ("shotfile", C.c_char * 224),
                ("geomfile", C.c_char * 224), ("jobname", C.c_char * 256), ("tmppath", C.c_char * 512)]


class Geometry(C.Structure):
    _fields_ = [("nsrc", C.c_int), ("nrec", C.POINTER(C.c_int)), ("src", C.POINTER(Coord)),
                ("rec", C.POINTER(C.POINTER(Coord)))]


class Stats(C.Structure):
    _fields_ = [("loop_ms", C.c_double), ("cell_updates", C.c_double), ("gcells_per_s", C.c_double),
                ("kernel_launches", C.c_int), ("graph_used", C.c_int), ("grad_segment", C.c_int),
                ("variant", C.c_int), ("block", C.c_int), ("stages", C.c_int), ("seg_len", C.c_int),
                ("autotuned", C.c_int), ("alg_bytes", C.c_double), ("sweep_ms", C.c_double),
                ("recompute_ms", C.c_double), ("adjoint_ms", C.c_double), ("task_order", C.c_int)]


# Every symbol include/seis2d.h declares, with its ctypes signature.
SIGNATURES = {
    "s2d_abi_version": ([], C.c_int),
    "s2d_create": ([C.POINTER(C.c_void_p), C.c_int], C.c_int),
    "s2d_destroy": ([C.c_void_p], None),
    "s2d_last_error": ([C.c_void_p], C.c_char_p),
    "s2d_derive_steps": ([C.POINTER(Wave), C.POINTER(Steps)], C.c_int),
    "s2d_set_option": ([C.c_void_p, C.c_char_p, C.c_long], C.c_int),
    "s2d_model_create": ([C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                          C.c_void_p, C.c_void_p, C.c_uint, C.POINTER(C.c_int)], C.c_int),
    "s2d_model_destroy": ([C.c_void_p, C.c_int], C.c_int),
    "s2d_forward": ([C.c_void_p, C.POINTER(Shot), C.c_int, C.POINTER(Wave), C.POINTER(C.c_double), C.c_int,
                     C.c_int, C.c_int, C.c_void_p, C.c_uint, C.POINTER(Stats)], C.c_int),
    "s2d_gradient": ([C.c_void_p, C.POINTER(Shot), C.c_int, C.POINTER(Wave), C.POINTER(C.c_double), C.c_int,
                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.c_uint, C.POINTER(Stats)], C.c_int),
    "s2d_jobcard_read": ([C.c_char_p, C.POINTER(JobCard), C.c_char_p, C.c_size_t], C.c_int),
    "s2d_geometry_read": ([C.POINTER(JobCard), C.POINTER(Geometry), C.c_char_p, C.c_size_t], C.c_int),
    "s2d_geometry_free": ([C.POINTER(Geometry)], None),
    "s2d_check_stability": ([C.POINTER(JobCard), C.c_float, C.c_float, C.c_char_p, C.c_size_t], C.c_int),
    "s2d_run_jobcard": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t],
                        C.c_int),
    "s2d_workload": ([C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "s2d_run_jobcard_rank": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              C.c_char_p, C.c_size_t], C.c_int),
    "s2d_forward_static": ([C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p,
                            C.POINTER(Wave), C.POINTER(Shot), C.c_void_p, C.c_uint, C.c_void_p, C.c_char_p,
                            C.c_size_t], C.c_int),
}

_lib = None


class Seis2dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib():
    """The loaded library; raises if the CUDA extension has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m seis2d_b200.build` "
                "(the modelling path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        if L.s2d_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI {L.s2d_abi_version()}, these bindings want {ABI_VERSION}: "
                               "rebuild it with `python -m seis2d_b200.build`")
        _lib = L
    return _lib
