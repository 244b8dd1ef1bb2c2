"""CPU tests of the multi-rank scatter split over gloo, world_size 2.

Crystal scatter at (d, v) reads PE[k, v] for every crystal k at the same voxel v, so ranks
that own blocks of voxel columns (sharding.voxel_block) compute their own PE columns and
exchange nothing.  The rank-local computation here is the CPU oracle (the FP32 restatement of
the reference's PE and scatter kernels), standing in for the device: each rank fills only its
own PE columns, and the gathered scatter columns must equal the single-process matrix."""
import os
import socket

import numpy as np

from conftest import geometry, oracle, sharding_module


def _columns(geo, v0, nv):
    pe = np.zeros((geo.n_det, geo.n_vox), dtype=np.float32)       # only this rank's columns are filled
    pe[:, v0:v0 + nv] = oracle.pe(geo, prec=32, v0=v0, nv=nv).astype(np.float32)
    bc = oracle.bitmap_crystal(geo)
    bh = oracle.bitmap_collimator(geo)
    s = oracle.scatter(geo, pe, "crystal", bc, prec=32, v0=v0, nv=nv)
    s = s + oracle.scatter(geo, pe, "collimator", bh, prec=32, v0=v0, nv=nv)
    return s


def _geo():
    return geometry.mini(seed=41, rotated=True, nvox=(5, 3, 1), ncry=(4, 3), nholes=4)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    geo = _geo()
    v0, nv = sharding_module().voxel_block(geo.n_vox, rank, world)
    sizes = [sharding_module().voxel_block(geo.n_vox, r, world)[1] for r in range(world)]
    width = max(sizes)                          # gloo gathers equal shapes: pad, then trim
    cols = torch.zeros((geo.n_det, width), dtype=torch.float64)
    cols[:, :nv] = torch.from_numpy(_columns(geo, v0, nv))
    parts = [torch.zeros((geo.n_det, width), dtype=torch.float64) for _ in sizes]
    dist.all_gather(parts, cols)                # the test's check only; the split itself needs none
    if rank == 0:
        q.put(torch.cat([p[:, :n] for p, n in zip(parts, sizes)], 1).numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_voxel_blocks_cover_columns_once():
    sh = sharding_module()
    for n, w in ((2304, 2), (2304, 8), (15, 4), (3, 8)):
        cols = []
        for r in range(w):
            b, c = sh.voxel_block(n, r, w)
            cols.extend(range(b, b + c))
        assert cols == list(range(n))


def test_two_rank_scatter_columns_equal_the_single_process_matrix():
    import torch.multiprocessing as mp
    geo = _geo()
    full = _columns(geo, 0, geo.n_vox)
    assert full.max() > 0
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    got = q.get()
    assert np.array_equal(got, full)
