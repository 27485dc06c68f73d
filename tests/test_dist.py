"""Multi-rank host logic of the N>1 path on CPU: two gloo ranks split a
sinogram stack into slice ranges, reconstruct their own ranges (here with the
oracle, standing in for the GPU), reduce timings over ranks and gather the
volume to rank 0, which must equal the single-process reconstruction."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from ufob import dist as udist


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, stack, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    ctx = udist.init(backend="gloo", timeout_s=60)
    try:
        assert (ctx.rank, ctx.world) == (rank, world)
        mx = ctx.max_over_ranks(10.0 * (rank + 1))
        sm = ctx.sum_over_ranks(rank + 1)
        start, stop = udist.slice_range(stack.shape[0], rank, world)
        s2, e2, vol = udist.reconstruct_sharded(
            ctx, stack, lambda sub: oracle.backproject(np.asarray(sub)).astype(np.float32), gather=True)
        # rank 0 receives the whole volume, the others keep nothing
        assert (s2, e2) == ((0, stack.shape[0]) if rank == 0 else (start, stop))
        ctx.barrier()
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), np.array([mx, sm, start, stop]))
        if rank == 0:
            np.save(os.path.join(out_dir, "vol.npy"), vol.numpy())
        else:
            assert vol is None
    finally:
        udist.finish(ctx)


@pytest.mark.parametrize("nz", [5, 8])
def test_two_gloo_ranks_reconstruct_and_gather(tmp_path, nz):
    rng = np.random.default_rng(nz)
    stack = rng.standard_normal((nz, 24, 32)).astype(np.float32)
    mp.spawn(_worker, args=(2, _free_port(), stack, str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    assert r0[0] == r1[0] == 20.0 and r0[1] == r1[1] == 3.0
    # contiguous, balanced, complete
    assert r0[2] == 0 and r0[3] == r1[2] and r1[3] == nz and abs((r0[3] - r0[2]) - (r1[3] - r1[2])) <= 1
    ref = oracle.backproject(stack).astype(np.float32)
    assert np.array_equal(np.load(tmp_path / "vol.npy"), ref)


def test_slice_range_partitions():
    for n in (0, 1, 7, 2048):
        for world in (1, 2, 3, 8):
            ranges = [udist.slice_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_single_process_context_is_a_no_op():
    ctx = udist.Ctx()
    assert ctx.max_over_ranks(3.5) == 3.5 and ctx.sum_over_ranks(2) == 2
    ctx.barrier()
    start, stop, vol = udist.reconstruct_sharded(ctx, np.zeros((3, 4, 4)), lambda s: s + 1, gather=True)
    assert (start, stop) == (0, 3) and vol.shape == (3, 4, 4)


CONE = {"source-position-y": -120.0, "detector-position-y": 40.0, "center-position-x": 16.0,
        "center-position-z": 6.0}


def _volume_worker(rank, world, port, proj, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    ctx = udist.init(backend="gloo", timeout_s=60)
    try:
        n = proj.shape[0]
        a, b = udist.slice_range(n, rank, world)
        z0, z1, vol = udist.reconstruct_volume_sharded(
            ctx, torch.from_numpy(proj[a:b]), n, (-4.0, 4.0, 1.0),
            lambda p: oracle.fft_filter_ifft(np.asarray(p)).astype(np.float32),
            lambda allp, reg: oracle.general_backproject(np.asarray(allp), n, region=reg, **CONE).astype(np.float32),
            gather=True)
        assert (z0, z1) == ((0, 8) if rank == 0 else udist.slice_range(8, rank, world))
        if rank == 0:
            np.save(os.path.join(out_dir, "vol.npy"), vol.numpy())
        else:
            assert vol is None
    finally:
        udist.finish(ctx)


@pytest.mark.parametrize("n", [12, 13])
def test_two_gloo_ranks_cone_volume_split_along_z(tmp_path, n):
    """Each rank filters its share of the projections, one all-gather exchanges them, each rank
    backprojects its z range; rank 0's gathered volume equals the one-process reconstruction."""
    rng = np.random.default_rng(n)
    proj = rng.standard_normal((n, 12, 32)).astype(np.float32)
    mp.spawn(_volume_worker, args=(2, _free_port(), proj, str(tmp_path)), nprocs=2, join=True)
    ref = oracle.general_backproject(oracle.fft_filter_ifft(proj).astype(np.float32), n, region=(-4.0, 4.0, 1.0),
                                     **CONE).astype(np.float32)
    np.testing.assert_array_equal(np.load(tmp_path / "vol.npy"), ref)


def test_volume_sharded_single_process():
    ctx = udist.Ctx()
    proj = torch.zeros((3, 4, 8))
    z0, z1, vol = udist.reconstruct_volume_sharded(ctx, proj, 3, (0.0, 5.0, 1.0), lambda p: p + 1,
                                                   lambda allp, reg: torch.full((round((reg[1] - reg[0]) / reg[2] + 0.5), 2, 2), float(allp.sum())))
    assert (z0, z1) == (0, 5) and vol.shape == (5, 2, 2) and float(vol[0, 0, 0]) == 96.0
    with pytest.raises(ValueError):
        udist.reconstruct_volume_sharded(ctx, proj[:2], 3, (0.0, 5.0, 1.0), lambda p: p, lambda a, r: a)
