"""Python host API over the C ABI (include/seis2d.h).

Mirrors the reference's modelling seam (``modelling_module``,
src/src_cpu/modelling.h:106) with explicit arguments instead of globals:

    ctx = Context(device=0)
    m = ctx.model(vp, rho, dx, dz, nb=32)          # [nx][nz] float32
    seis = ctx.forward([Shot(m, (sx, sz), rec_xz)], Wave(T, dt, data_dt, f))
    # seis[s] is [nrec][real_nt] float32, the reference's file layout

Arrays may be numpy (host) or CUDA torch tensors (device); torch is needed
only for the latter.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib as L


@dataclass(frozen=True)
class Wave:
    """``wave_t`` (src/src_cpu/modelling.h:27-31): seconds and Hz."""
    rec_len: float
    fd_dt: float
    real_dt: float
    dom_freq: float

    def c(self) -> L.Wave:
        return L.Wave(self.rec_len, self.fd_dt, self.real_dt, self.dom_freq)


def derive_steps(wave: Wave) -> dict:
    out = L.Steps()
    rc = L.lib().s2d_derive_steps(C.byref(wave.c()), C.byref(out))
    if rc:
        raise L.Seis2dError(rc, "bad wave parameters")
    return {"fd_nt": out.fd_nt, "real_nt": out.real_nt, "dt_factor": out.dt_factor, "nts": out.nts}


class Model:
    def __init__(self, ctx: "Context", mid: int, nx: int, nz: int, dx: float, dz: float, nb: int):
        self.ctx, self.id, self.nx, self.nz, self.dx, self.dz, self.nb = ctx, mid, nx, nz, dx, dz, nb

    @property
    def padded_cells(self) -> int:
        return (self.nx + 2 * self.nb) * (self.nz + 2 * self.nb)

    def release(self):
        if self.ctx is not None and self.ctx._h:
            L.lib().s2d_model_destroy(self.ctx._h, self.id)
        self.ctx = None


@dataclass
class Shot:
    model: Model
    src: Tuple[float, float]
    rec: np.ndarray  # (nrec, 2) metres: x, z


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


class Context:
    """One CUDA device; owns the device memory of its models and shots."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        rc = L.lib().s2d_create(C.byref(self._h), int(device))
        if rc:
            raise L.Seis2dError(rc, "s2d_create failed (no usable CUDA device?)")
        self.device = device
        self.last_stats: Optional[L.Stats] = None

    def _check(self, rc: int):
        if rc:
            raise L.Seis2dError(rc, L.lib().s2d_last_error(self._h).decode())

    def close(self):
        if self._h:
            L.lib().s2d_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, key: str, value: int):
        """Step-kernel tuning knob (see s2d_set_option in include/seis2d.h)."""
        self._check(L.lib().s2d_set_option(self._h, key.encode(), int(value)))

    def model(self, vp, rho, dx: float, dz: float, nb: int = 32, free_surface: bool = False,
              fd_order: int = 4) -> Model:
        """Upload a ``[nx][nz]`` model (numpy or CUDA tensor, float32).

        ``free_surface``: the first model row is a pressure-release surface
        (kappa held at 0 on it and on the sponge rows above it), what the job
        card's ``"Free surface" : "1"`` asks for; the reference parses that key
        and ignores it, so the default keeps its results.
        ``fd_order``: 4 (the reference's operator) or 8 (the staggered
        8th-order operator, job card ``"Order of FD Operator" : "8"``, which
        the reference parses and never runs); shots of one call share it."""
        if fd_order not in (4, 8):
            raise ValueError("fd_order must be 4 or 8")
        flags = L.S2D_MODEL_FREE_SURFACE if free_surface else 0
        if fd_order == 8:
            flags |= L.S2D_MODEL_ORDER8
        if _is_torch(vp):
            import torch
            assert vp.is_cuda and rho.is_cuda and vp.dtype == torch.float32 and rho.dtype == torch.float32
            vp, rho = vp.contiguous(), rho.contiguous()
            nx, nz = vp.shape
            pv, pr = C.c_void_p(vp.data_ptr()), C.c_void_p(rho.data_ptr())
            flags |= L.S2D_MODEL_DEVICE
            keep = (vp, rho)
        else:
            vp = np.ascontiguousarray(vp, np.float32)
            rho = np.ascontiguousarray(rho, np.float32)
            nx, nz = vp.shape
            pv, pr = C.c_void_p(vp.ctypes.data), C.c_void_p(rho.ctypes.data)
            keep = (vp, rho)
        if tuple(rho.shape) != (nx, nz):
            raise ValueError("vp and rho shapes differ")
        mid = C.c_int()
        self._check(L.lib().s2d_model_create(self._h, int(nx), int(nz), float(dx), float(dz), int(nb),
                                             pv, pr, flags, C.byref(mid)))
        del keep
        return Model(self, mid.value, int(nx), int(nz), float(dx), float(dz), int(nb))

    def forward(self, shots: Sequence[Shot], wave: Wave, wavelet: Optional[np.ndarray] = None,
                kt_begin: int = 0, kt_count: int = 0, out=None, plain: bool = False,
                graph: bool = True, sync: bool = True):
        """Run the FD loop; returns ``out`` (allocated if None).

        ``out`` is one flat float32 buffer of ``sum(nrec_s) * real_nt`` samples
        (numpy for host output, CUDA tensor for device output); the returned
        value is split per shot as ``[nrec_s][real_nt]`` views when ``out`` was
        not given.
        """
        steps = derive_steps(wave)
        nt = steps["real_nt"]
        cshots = (L.Shot * len(shots))()
        keep = []
        total = 0
        for i, s in enumerate(shots):
            rec = np.ascontiguousarray(s.rec, np.float32).reshape(-1, 2)
            keep.append(rec)
            cshots[i].model_id = s.model.id
            cshots[i].src = L.Coord(float(s.src[0]), float(s.src[1]))
            cshots[i].nrec = rec.shape[0]
            cshots[i].rec = rec.ctypes.data_as(C.POINTER(L.Coord))
            total += rec.shape[0]
        flags = 0
        given = out is not None
        if out is None:
            out = np.zeros(total * nt, np.float32)
        if _is_torch(out):
            assert out.is_cuda and out.numel() >= total * nt
            flags |= L.S2D_SEIS_DEVICE
            ptr = C.c_void_p(out.data_ptr())
        else:
            assert out.dtype == np.float32 and out.size >= total * nt and out.flags.c_contiguous
            ptr = C.c_void_p(out.ctypes.data)
        if plain:
            flags |= L.S2D_PLAIN
        if not graph:
            flags |= L.S2D_NO_GRAPH
        if sync:
            flags |= L.S2D_SYNC
        wp, nw = None, 0
        if wavelet is not None:
            wavelet = np.ascontiguousarray(wavelet, np.float64)
            keep.append(wavelet)
            wp, nw = wavelet.ctypes.data_as(C.POINTER(C.c_double)), wavelet.size
        st = L.Stats()
        self._check(L.lib().s2d_forward(self._h, cshots, len(shots), C.byref(wave.c()), wp, nw,
                                        int(kt_begin), int(kt_count), ptr, flags, C.byref(st)))
        self.last_stats = st
        if given:
            return out
        res, off = [], 0
        for s in shots:
            n = np.asarray(s.rec).reshape(-1, 2).shape[0]
            res.append(out[off * nt:(off + n) * nt].reshape(n, nt))
            off += n
        return res


class GradientResult:
    """Result of Context.gradient: dJ/dvp and dJ/drho ([nx][nz]), the
    misfit (misfit mode), the forward seismograms (if asked) and dJ/dw per
    shot and FD step."""

    def __init__(self, grad_vp, grad_rho, misfit, seis, grad_wavelet, stats):
        self.grad_vp, self.grad_rho, self.misfit = grad_vp, grad_rho, misfit
        self.seis, self.grad_wavelet, self.stats = seis, grad_wavelet, stats


def _gradient(self: "Context", shots: Sequence[Shot], wave: Wave, data, misfit: bool = False,
              wavelet: Optional[np.ndarray] = None, grad_vp=None, grad_rho=None, want_seis: bool = False,
              graph: bool = True) -> GradientResult:
    """FWI gradient of the shots (one model).  ``data`` is dJ/d(seis) or, with
    ``misfit=True``, the observed seismograms (J = 0.5 ||d - data||^2); same
    flat layout as ``forward``'s output.  numpy arrays are host buffers; CUDA
    tensors are device buffers (``grad_vp``/``grad_rho`` given as CUDA tensors
    receive the gradient in place)."""
    steps = derive_steps(wave)
    nt, fd_nt = steps["real_nt"], steps["fd_nt"]
    m = shots[0].model
    cshots = (L.Shot * len(shots))()
    keep = []
    total = 0
    for i, s in enumerate(shots):
        rec = np.ascontiguousarray(s.rec, np.float32).reshape(-1, 2)
        keep.append(rec)
        cshots[i] = L.Shot(s.model.id, L.Coord(float(s.src[0]), float(s.src[1])), rec.shape[0],
                           rec.ctypes.data_as(C.POINTER(L.Coord)))
        total += rec.shape[0]
    flags = L.S2D_GRAD_MISFIT if misfit else 0
    if not graph:
        flags |= L.S2D_NO_GRAPH
    if _is_torch(data):
        assert data.is_cuda and data.numel() >= total * nt
        flags |= L.S2D_SEIS_DEVICE
        dptr = C.c_void_p(data.data_ptr())
        seis = None
        if want_seis:
            import torch
            seis = torch.empty(total * nt, dtype=torch.float32, device=data.device)
    else:
        data = np.ascontiguousarray(data, np.float32).reshape(-1)
        assert data.size >= total * nt
        keep.append(data)
        dptr = C.c_void_p(data.ctypes.data)
        seis = np.zeros(total * nt, np.float32) if want_seis else None
    sptr = None
    if seis is not None:
        sptr = C.c_void_p(seis.data_ptr() if _is_torch(seis) else seis.ctypes.data)
    if grad_vp is not None and _is_torch(grad_vp):
        flags |= L.S2D_GRAD_DEVICE
        gv, gr = grad_vp, grad_rho
        gvp, grp = C.c_void_p(gv.data_ptr()), C.c_void_p(gr.data_ptr())
    else:
        gv = np.zeros((m.nx, m.nz), np.float32)
        gr = np.zeros((m.nx, m.nz), np.float32)
        gvp, grp = C.c_void_p(gv.ctypes.data), C.c_void_p(gr.ctypes.data)
    wp, nw = None, 0
    if wavelet is not None:
        wavelet = np.ascontiguousarray(wavelet, np.float64)
        keep.append(wavelet)
        wp, nw = wavelet.ctypes.data_as(C.POINTER(C.c_double)), wavelet.size
    gw = np.zeros((len(shots), fd_nt), np.float64)
    mis = C.c_double(0.0)
    st = L.Stats()
    self._check(L.lib().s2d_gradient(self._h, cshots, len(shots), C.byref(wave.c()), wp, nw, dptr, gvp, grp,
                                     sptr, C.byref(mis), gw.ctypes.data_as(C.POINTER(C.c_double)), flags,
                                     C.byref(st)))
    self.last_stats = st
    return GradientResult(gv, gr, mis.value if misfit else None, seis, gw, st)


Context.gradient = _gradient


def modelling_module(vp: np.ndarray, rho: np.ndarray, dx: float, dz: float, wave: Wave,
                     geometry: Sequence[Tuple[Tuple[float, float], np.ndarray]], nb: int = 32,
                     device: int = 0, plain: bool = False, free_surface: bool = False,
                     fd_order: int = 4) -> List[np.ndarray]:
    """The reference seam with explicit arguments: every shot of
    ``geometry`` = ``[((sx, sz), rec_xz), ...]`` on one model, returning the
    per-shot ``[nrec][real_nt]`` seismograms the reference writes to disk
    (src/src_cpu/cpumodelling.cpp:158-383)."""
    with Context(device) as ctx:
        m = ctx.model(vp, rho, dx, dz, nb, free_surface=free_surface, fd_order=fd_order)
        shots = [Shot(m, src, np.asarray(rec, np.float32)) for src, rec in geometry]
        return [s.copy() for s in ctx.forward(shots, wave, plain=plain)]
