"""The multi-rank path on CPU: world_size 2 over gloo.  Each rank filters its
share of the blocks of a tile walk (through the oracle, as the reference result) and
the gathered result equals the whole-image filter: the work list shards with
no collective on the data path."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from lucem_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _schedule(dims, block, halo):
    # crates/lucem-core/src/tiling.rs:54-78 (host rule; the C ABI has the same one)
    import lucem_b200 as lb

    return lb.schedule(dims, block, halo)


def _rank_main(rank, world, port, out_dir):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    import torch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        H, W = 150, 230
        x = (np.arange(H * W, dtype=np.float32).reshape(H, W) % 97) * 0.5
        blocks = _schedule((1, H, W), (1, 64, 64), (0, 12, 12))
        mine = shard.shard(blocks, rank, world, shard.block_cost)
        part = np.zeros((H, W), np.float32)
        for b in mine:
            ry, rx, rh, rw = b.read_origin[1], b.read_origin[2], b.read_size[1], b.read_size[2]
            y = O.gaussian_blur(np.ascontiguousarray(x[ry:ry + rh, rx:rx + rw]), [2.0])
            oy, ox = b.origin[1] - ry, b.origin[2] - rx
            part[b.origin[1]:b.origin[1] + b.size[1], b.origin[2]:b.origin[2] + b.size[2]] = \
                y[oy:oy + b.size[1], ox:ox + b.size[2]]
        t = torch.from_numpy(part)
        dist.all_reduce(t)  # each pixel is owned by exactly one rank
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), t.numpy())
            np.save(os.path.join(out_dir, "whole.npy"), O.gaussian_blur(x, [2.0]))
    finally:
        dist.destroy_process_group()


def test_split_balanced_covers_everything_once():
    costs = [5, 1, 1, 1, 9, 2, 2, 3]
    for world in (1, 2, 3, 8, 10):
        b = shard.split_balanced(costs, world)
        assert b[0] == 0 and b[-1] == len(costs) and len(b) == world + 1
        assert all(b[i] <= b[i + 1] for i in range(world))
    items = list(range(17))
    got = sum((shard.shard(items, r, 4) for r in range(4)), [])
    assert got == items


def test_two_ranks_gloo_tile_walk_equals_whole_image(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    gathered = np.load(tmp_path / "gathered.npy")
    whole = np.load(tmp_path / "whole.npy")
    assert np.abs(gathered - whole).max() < 1e-3


def _psf_fit_rank(rank, world, port, out_dir):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle as O
    import torch

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        vols = [rng.uniform(0.5, 2.0, (6, 10, 9)) for _ in range(5)]
        ws = [rng.standard_normal((6, 10, 9)) for _ in range(5)]
        psf = rng.uniform(0.2, 1.0, (3, 3, 3))
        mine = shard.shard(list(range(5)), rank, world, lambda i: float(vols[i].size))
        g = np.zeros(psf.shape)
        for i in mine:
            g += O.richardson_lucy_backward_fft64(vols[i], psf, ws[i], num_iter=3, filter_epsilon=1e-6)[0]
        t = torch.from_numpy(g)
        shard.allreduce_psf_grad(t)
        if rank == 0:
            np.save(os.path.join(out_dir, "dp.npy"), t.numpy())
            whole = sum(O.richardson_lucy_backward_fft64(v, psf, w, num_iter=3, filter_epsilon=1e-6)[0]
                        for v, w in zip(vols, ws))
            np.save(os.path.join(out_dir, "single.npy"), whole)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo_psf_gradient_allreduce(tmp_path):
    """Data-parallel PSF fit: each rank's share of the volumes, one all-reduce
    of the PSF gradient, equal to the single-process sum."""
    port = _free_port()
    mp.start_processes(_psf_fit_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    dp = np.load(tmp_path / "dp.npy")
    single = np.load(tmp_path / "single.npy")
    assert np.allclose(dp, single, rtol=1e-12, atol=1e-15)
