"""``torch.autograd.Function`` over the C ABI: seismograms as a
differentiable function of vp and rho.

    seis = modelled_seismograms(vp, rho, shots_xz, wave, dx, dz, nb)   # CUDA tensors
    loss = 0.5 * ((seis - d_obs) ** 2).sum()
    loss.backward()                      # vp.grad, rho.grad from the hand-written adjoint

forward runs s2d_forward; backward runs s2d_gradient with the incoming
gradient as the adjoint source (it recomputes the forward wavefield with
checkpoints).  Both stay on the device.
"""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np
import torch

from .api import Context, Shot, Wave, derive_steps

_contexts = {}


def _context(device: torch.device) -> Context:
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _contexts:
        _contexts[idx] = Context(idx)
    return _contexts[idx]


class ForwardModelling(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vp, rho, geometry, wave, dx, dz, nb):
        assert vp.is_cuda and rho.is_cuda and vp.dtype == torch.float32 and rho.dtype == torch.float32
        sctx = _context(vp.device)
        vp_c, rho_c = vp.detach().contiguous(), rho.detach().contiguous()
        m = sctx.model(vp_c, rho_c, dx, dz, nb)
        shots = [Shot(m, src, np.asarray(rec, np.float32)) for src, rec in geometry]
        nt = derive_steps(wave)["real_nt"]
        total = sum(np.asarray(rec).reshape(-1, 2).shape[0] for _, rec in geometry)
        out = torch.empty(total * nt, dtype=torch.float32, device=vp.device)
        sctx.forward(shots, wave, out=out)
        m.release()
        ctx.save_for_backward(vp_c, rho_c)
        ctx.meta = (geometry, wave, dx, dz, nb)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        vp, rho = ctx.saved_tensors
        geometry, wave, dx, dz, nb = ctx.meta
        sctx = _context(vp.device)
        m = sctx.model(vp, rho, dx, dz, nb)
        shots = [Shot(m, src, np.asarray(rec, np.float32)) for src, rec in geometry]
        gvp = torch.empty_like(vp)
        grho = torch.empty_like(rho)
        sctx.gradient(shots, wave, grad_out.detach().contiguous(), grad_vp=gvp, grad_rho=grho)
        m.release()
        return gvp, grho, None, None, None, None, None


def modelled_seismograms(vp: torch.Tensor, rho: torch.Tensor,
                         geometry: Sequence[Tuple[Tuple[float, float], np.ndarray]], wave: Wave,
                         dx: float, dz: float, nb: int = 32) -> torch.Tensor:
    """Flat float32 tensor of all shots' ``[nrec][real_nt]`` seismograms."""
    return ForwardModelling.apply(vp, rho, list(geometry), wave, dx, dz, nb)
