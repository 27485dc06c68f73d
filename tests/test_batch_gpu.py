"""Uneven batch of parallel-beam reconstructions in one graph launch
(persistent filter and backprojection kernels over work queues, autotuned
tile shape) against the FP64 oracle of each job's own graph
`fft size-x=N ! filter ! ifft crop-width=W ! backproject`."""
import math
import os

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu

SHAPES = [(64, 90), (128, 200), (96, 77), (256, 181), (64, 300), (160, 45), (32, 16), (128, 512)]


def _jobs(seed):
    rng = np.random.default_rng(seed)
    jobs, refs = [], []
    for i, (W, P) in enumerate(SHAPES):
        ell = oracle.random_ellipses(seed * 100 + i)
        axis = W / 2.0 + (0.25 if i % 3 == 1 else 0.0)
        step = math.pi / P
        offset = 0.1 * (i % 2)
        sino = oracle.ellipse_sinogram(ell, W, offset + np.arange(P) * step, axis=axis).astype(np.float32)
        sino += 0.01 * rng.standard_normal(sino.shape).astype(np.float32)
        N = 1 << (W - 1).bit_length()
        ref = oracle.backproject(oracle.fft_filter_ifft(sino, size_x=N, crop_width=W).astype(np.float32),
                                 axis_pos=axis, angle_step=step, angle_offset=offset)
        d = torch.from_numpy(sino).cuda()
        out = torch.zeros((W, W), dtype=torch.float32, device="cuda")
        jobs.append(dict(sino=d, out=out, axis_pos=axis, angle_step=step, angle_offset=offset))
        refs.append(ref)
    return jobs, refs


@pytest.fixture(autouse=True)
def tune_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("UFOB_TUNE_CACHE", str(tmp_path / "tune.txt"))


@pytest.mark.parametrize("storage,tol", [(ufob.F32, 1e-5), (ufob.F16, 1e-3)])
def test_batch_matches_oracle(cuda, storage, tol):
    jobs, refs = _jobs(1)
    b = ufob.Batch(storage=storage)
    b.run(jobs)
    torch.cuda.synchronize()
    ufob.device_status()
    assert 0 <= b.variant() < 8
    for j, ref in zip(jobs, refs):
        assert oracle.rel_l2(j["out"].cpu().numpy(), ref) < tol


@pytest.mark.parametrize("storage,tol", [(ufob.F32, 1e-5), (ufob.F16, 1e-3), (ufob.BF16, 8e-3)])
def test_every_tile_variant_matches_oracle(cuda, storage, tol):
    """Each tile shape the autotuner may pick (pinned one by one), on the uneven jobs plus a
    1536-angle job, which turns on the blocked-Kahan sums of the 16-bit forms."""
    jobs, refs = _jobs(4)
    W, P = 128, 1536
    ell = oracle.random_ellipses(4321)
    sino = oracle.ellipse_sinogram(ell, W, np.arange(P) * math.pi / P).astype(np.float32)
    refs.append(oracle.backproject(oracle.fft_filter_ifft(sino, size_x=W, crop_width=W).astype(np.float32)))
    jobs.append(dict(sino=torch.from_numpy(sino).cuda(), out=torch.zeros((W, W), device="cuda")))
    b = ufob.Batch(storage=storage)
    assert ufob.Batch.variants() == 8
    for v in range(ufob.Batch.variants()):
        b.set_variant(v)
        for j in jobs:
            j["out"].zero_()
        b.run(jobs)
        torch.cuda.synchronize()
        ufob.device_status()
        assert b.variant() == v
        for j, ref in zip(jobs, refs):
            assert oracle.rel_l2(j["out"].cpu().numpy(), ref) < tol, (v, j["sino"].shape)
    b.set_variant(-1)


def test_batch_graph_replay_and_change(cuda):
    jobs, refs = _jobs(2)
    b = ufob.Batch()
    b.run(jobs)
    for j in jobs:
        j["out"].zero_()
    b.run(jobs)  # replay of the captured graph
    torch.cuda.synchronize()
    for j, ref in zip(jobs, refs):
        assert oracle.rel_l2(j["out"].cpu().numpy(), ref) < 1e-5
    # new inputs in the same buffers: replay sees the new data
    jobs2, refs2 = _jobs(3)
    for j, j2 in zip(jobs, jobs2):
        j["sino"].copy_(j2["sino"])
    b.run(jobs[:])
    torch.cuda.synchronize()
    # geometry of jobs2 equals jobs (same shapes and props), so refs2 apply
    for j, ref in zip(jobs, refs2):
        assert oracle.rel_l2(j["out"].cpu().numpy(), ref) < 1e-5
    # a different batch (fewer jobs) re-captures
    b.run(jobs[:3])
    torch.cuda.synchronize()


def test_tuning_cache_written(cuda, tmp_path):
    jobs, _ = _jobs(4)
    b = ufob.Batch()
    b.run(jobs)
    torch.cuda.synchronize()
    path = os.environ["UFOB_TUNE_CACHE"]
    text = open(path).read()
    assert text.startswith("bp_batch:") and str(b.variant()) in text.split()[-1]


def test_batch_rejects_unaligned(cuda):
    sino = torch.zeros((10, 30), device="cuda")
    out = torch.zeros((30, 30), device="cuda")
    with pytest.raises(ufob.UfobError):
        ufob.Batch().run([dict(sino=sino, out=out)])
