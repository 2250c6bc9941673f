"""Shots over several ranks (seis2d_b200.sharding) on the CPU: the shot
partition against the reference's calculate_workload rule, and the gradient
sum of a 2-rank gloo job (each rank's block computed by the FP64 oracle)
against the sum over all shots in one process."""
import os
import socket

import numpy as np
import pytest

from oracle import oracle as O


def reference_workload(nsrc, size):
    """calculate_workload (workload.cpp:34-48), restated."""
    div, mod = nsrc // size, nsrc % size
    out, start = [], 0
    for i in range(size):
        n = div + 1 if i < mod else div
        out.append((start, n))
        start += n
    return out


@pytest.mark.parametrize("nsrc,size", [(1, 1), (7, 1), (8, 8), (9, 8), (64, 8), (65, 8), (100, 7), (3, 2)])
def test_shot_block_is_the_reference_partition(nsrc, size):
    from seis2d_b200.sharding import shot_block
    got = [shot_block(nsrc, r, size) for r in range(size)]
    assert got == reference_workload(nsrc, size)
    assert sum(n for _, n in got) == nsrc


def test_fewer_shots_than_ranks_is_an_error():
    from seis2d_b200._lib import Seis2dError
    from seis2d_b200.sharding import shot_block
    with pytest.raises(Seis2dError, match="-8"):
        shot_block(3, 0, 4)
    with pytest.raises(Seis2dError):
        shot_block(8, 8, 8)


def test_forward_block_takes_the_ranks_shots():
    from seis2d_b200.sharding import forward_block

    class Recorder:
        def forward(self, shots, wave, **kw):
            return list(shots)

    # outside a process group: rank 0 of 1 takes every shot
    first, got = forward_block(Recorder(), list(range(5)), None)
    assert first == 0 and got == [0, 1, 2, 3, 4]


# ---- 2-rank gloo job: FWI gradient summed over ranks ----

NX, NZ, NB, D = 26, 18, 8, 10.0
T, DT, F = 0.12, 0.001, 25.0
SHOTS = [(60.0, 20.0), (110.0, 20.0), (150.0, 30.0), (200.0, 20.0), (230.0, 40.0)]


def _setup():
    x = np.linspace(0, 1, NX)[:, None]
    z = np.linspace(0, 1, NZ)[None, :]
    vp = (1800 + 700 * z + 60 * np.sin(5 * x)).astype(np.float32)
    rho = (1400 + 300 * z + 0 * x).astype(np.float32)
    vp_true = vp.copy()
    vp_true[10:16, 6:12] += 120.0
    rx = np.arange(1, NX - 1, 2) * D
    rec = np.stack([rx, np.full(rx.size, 20.0)], 1).astype(np.float32)
    p = O.Params(NX, NZ, NB, D, D, T, DT, DT, F)
    return vp, rho, vp_true, rec, p


def _observed(vp_true, rho, rec, p):
    return [O.gradient(p, vp_true, rho, s, rec[:, 0], rec[:, 1], None)["seis64"] for s in SHOTS]


def _local_gradient(vp, rho, rec, p):
    def fn(block, data_block):
        gv = np.zeros((NX, NZ))
        gr = np.zeros((NX, NZ))
        mis = 0.0
        for s, d in zip(block, data_block):
            seis = O.gradient(p, vp, rho, s, rec[:, 0], rec[:, 1], None)["seis64"]
            r = seis - d
            g = O.gradient(p, vp, rho, s, rec[:, 0], rec[:, 1], r)
            gv += g["grad_vp"]
            gr += g["grad_rho"]
            mis += 0.5 * float(np.sum(r * r))
        return gv, gr, mis
    return fn


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from seis2d_b200.sharding import gradient_allreduce, shot_block
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        vp, rho, vp_true, rec, p = _setup()
        dobs = _observed(vp_true, rho, rec, p)
        first, count = shot_block(len(SHOTS))
        gv, gr, mis = gradient_allreduce(None, SHOTS, None, dobs[first:first + count],
                                         local_gradient=_local_gradient(vp, rho, rec, p))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), gv=gv.numpy(), gr=gr.numpy(), mis=mis,
                 first=first, count=count)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_gradient_allreduce_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    vp, rho, vp_true, rec, p = _setup()
    dobs = _observed(vp_true, rho, rec, p)
    gv, gr, mis = _local_gradient(vp, rho, rec, p)(SHOTS, dobs)
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in (0, 1))
    assert (int(r0["first"]), int(r0["count"]), int(r1["first"]), int(r1["count"])) == (0, 3, 3, 2)
    for r in (r0, r1):   # every rank holds the sum over all shots
        assert O.rel_l2(r["gv"], gv) <= 1e-6
        assert O.rel_l2(r["gr"], gr) <= 1e-6
        assert abs(float(r["mis"]) - mis) <= 1e-9 * mis
    assert np.abs(gv).max() > 0
