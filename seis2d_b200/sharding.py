"""Shots over several GPUs: one process per GPU, ``torch.distributed`` for the
plumbing.  Replaces the reference's MPI master/worker distribution
(``src/src_cpu/workload.cpp:12-62``, ``modelling_master.cpp`` /
``modelling_worker.cpp``) and the per-device OpenMP team of the multi-GPU
backend (``src/src_gpu_multi/gpumodelling_multi.cu:292-420``, which needs
``ns % ndevices == 0``).

* Forward modelling shards with no collective: every rank models its
  contiguous block of shots (``shot_block``: the reference's
  ``calculate_workload`` rule) with the model replicated.
* The FWI gradient is one sum over shots: each rank's library call already
  sums its own shots on the GPU, then a single all-reduce (NCCL over NVLink on
  GPUs, gloo on CPU) adds the ranks' (dJ/dvp, dJ/drho, misfit) in one flat
  buffer.

Usage, launched as ``torchrun --nproc-per-node N script.py``::

    dist.init_process_group("nccl")
    ctx = Context(local_rank)
    first, n = shot_block(len(shots), rank, world)
    seis = forward_block(ctx, shots, wave)                # this rank's shots
    g = gradient_allreduce(ctx, shots, wave, dobs_block)   # summed over ranks
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L


def _group_rank_size(group=None) -> Tuple[int, int]:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def shot_block(nsrc: int, rank: Optional[int] = None, nranks: Optional[int] = None, group=None) -> Tuple[int, int]:
    """``(first, count)`` of rank ``rank``'s shots: contiguous blocks, the
    first ``nsrc % nranks`` ranks one shot longer (workload.cpp:34-48).
    Fewer shots than ranks is an error, as in the reference (workload.cpp:21-31,
    abort -8).  Rank and size default to the process group's."""
    if rank is None or nranks is None:
        r, n = _group_rank_size(group)
        rank = r if rank is None else rank
        nranks = n if nranks is None else nranks
    first, count = C.c_int(), C.c_int()
    rc = L.lib().s2d_workload(int(nsrc), int(nranks), int(rank), C.byref(first), C.byref(count))
    if rc:
        if nsrc < nranks:
            raise L.Seis2dError(rc, f"number of sources ({nsrc}) should be greater than or equal to the number "
                                    f"of ranks ({nranks}) (reference code -8)")
        raise L.Seis2dError(rc, f"bad rank {rank} of {nranks}")
    return first.value, count.value


def forward_block(ctx, shots: Sequence, wave, group=None, **kwargs):
    """Forward modelling of this rank's block of ``shots``; returns
    ``(first, seismograms)`` with the seismograms of shots
    ``first .. first + len - 1`` as ``Context.forward`` returns them.  No
    collective."""
    first, count = shot_block(len(shots), group=group)
    return first, ctx.forward(list(shots[first:first + count]), wave, **kwargs)


def gradient_allreduce(ctx, shots: Sequence, wave, data_block, misfit: bool = True, group=None,
                       local_gradient: Optional[Callable] = None, **kwargs):
    """FWI gradient over all ranks' shots: this rank's block (``data_block``
    holds the block's observed data, or its adjoint source with
    ``misfit=False``, in ``Context.forward``'s flat layout), then one
    all-reduce (sum) of ``[dJ/dvp, dJ/drho, misfit]``.

    ``local_gradient(block_shots, data_block) -> (grad_vp, grad_rho, misfit)``
    replaces the library call for the block (the CPU tests run the ranks on
    the oracle this way); by default it is ``ctx.gradient`` with device
    outputs.  Returns ``(grad_vp, grad_rho, misfit)`` as torch tensors on the
    rank's device (CPU for gloo) and a float; every rank gets the sum."""
    import torch
    import torch.distributed as dist
    first, count = shot_block(len(shots), group=group)
    block = list(shots[first:first + count])
    if local_gradient is None:
        m = block[0].model
        dev = torch.device("cuda", torch.cuda.current_device())
        gv = torch.zeros(m.nx, m.nz, dtype=torch.float32, device=dev)
        gr = torch.zeros_like(gv)
        res = ctx.gradient(block, wave, data_block, misfit=misfit, grad_vp=gv, grad_rho=gr, **kwargs)
        mis = res.misfit if misfit else 0.0
    else:
        gv, gr, mis = local_gradient(block, data_block)
        gv = torch.as_tensor(np.asarray(gv, np.float32) if not torch.is_tensor(gv) else gv)
        gr = torch.as_tensor(np.asarray(gr, np.float32) if not torch.is_tensor(gr) else gr)
    n = gv.numel()
    # one collective per gradient evaluation: images and misfit in one FP64
    # buffer (2 nx nz + 1 values, 7.7 MB for a 1201 x 401 model)
    flat = torch.empty(2 * n + 1, dtype=torch.float64, device=gv.device)
    flat[:n] = gv.reshape(-1)
    flat[n:2 * n] = gr.reshape(-1)
    flat[2 * n] = float(mis or 0.0)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    gv = flat[:n].reshape(gv.shape).to(torch.float32)
    gr = flat[n:2 * n].reshape(gr.shape).to(torch.float32)
    return gv, gr, float(flat[2 * n].item())


def run_jobcard_distributed(path: str, device: Optional[int] = None, nb: int = 32, naming: str = "cpu",
                            check_stability: bool = True, verbose: bool = False, group=None) -> Tuple[int, int]:
    """Every rank of the process group runs its block of the card's shots on
    its own GPU (``device`` defaults to the rank's local GPU) through the C
    host driver; returns the rank's ``(first, count)``."""
    import os
    from .driver import read_geometry, read_jobcard, run_jobcard
    rank, nranks = _group_rank_size(group)
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", "0"))
    nsrc = len(read_geometry(read_jobcard(path)))
    block = shot_block(nsrc, rank, nranks)
    run_jobcard(path, device=device, nb=nb, naming=naming, check_stability=check_stability, verbose=verbose,
                rank=rank, nranks=nranks)
    return block
