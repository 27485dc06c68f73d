"""The benchmarked workloads at their own shapes.

* One 32-slice group of the batched FBP (2048 detector bins x 1500 angles,
  noisy ellipsoid phantom) in plain FP32 and in FP16 slice-quad storage with
  blocked Kahan sums, against the FP64 oracle on a 256^2 region of four of its
  slices and, for the plain form, against the reference's own filter and
  backproject code compiled for the CPU (src/ufo-filter-task.c,
  src/ufo-backproject-task.c, src/kernels/backproject.cl) on the same region:
  the plain form must match the reference within 1e-4 relative L2.
* An uneven batch holding the widest jobs of that workload (1536 and 2048 bins,
  up to 1800 angles) next to small ones, each job against the oracle of its own
  graph `fft size-x=N ! filter ! ifft crop-width=W ! backproject`.
* A cone-beam general backprojection from 1024 projections into a reduced
  volume, three of its slices against the oracle of
  src/ufo-general-backproject-task.c's transform chain.
"""
import math

import numpy as np
import pytest
import torch

import oracle
import reference
import ufob

pytestmark = pytest.mark.gpu

I0 = 1.0e4


def _group(nz=32, P=1500, W=2048, total=2048, z0=1008, seed=2024):
    """nz slices of the full-size noisy stack starting at slice z0 (analytic
    ellipsoid line integrals, Beer-Lambert with I0 photons, Poisson noise)."""
    ell = oracle.random_ellipsoids(seed)
    scale = W / 2.0
    ell[:, 2] -= (z0 + 0.5 * nz - 0.5 * total) / scale
    s = ufob.phantom_stack(ell, W, P, nz)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    counts = torch.poisson(I0 * torch.exp(-s / scale), generator=gen)
    return (-torch.log(torch.clamp(counts, min=0.5) / I0) * scale).contiguous()


@pytest.fixture(scope="module")
def c1_group(cuda):
    stack = _group()
    W = stack.shape[-1]
    picks = [0, 11, 22, 31]
    rx, ry, side = 1100, 700, 256
    host = [stack[i].cpu().numpy() for i in picks]
    refs = [oracle.backproject(oracle.fft_filter_ifft(s).astype(np.float32), axis_pos=W / 2.0,
                               roi_x=rx, roi_y=ry, roi_width=side, roi_height=side) for s in host]
    return stack, picks, (rx, ry, side), host, refs


# FP32 bound: 1500 uncompensated FP32 sums per pixel of a noisy phantom (the plain form, as the
# reference sums); the FP16 forms (the default FP32 block sums, and blocked Kahan sums on request)
# are bounded by the FP16 rounding of the filtered cells
@pytest.mark.parametrize("storage,compensated,tol", [(ufob.F32, 0, 3e-5), (ufob.F16, 0, 1e-3), (ufob.F16, 1, 1e-3)])
def test_c1_group_vs_oracle(c1_group, storage, compensated, tol):
    stack, picks, (rx, ry, side), _, refs = c1_group
    W = stack.shape[-1]
    fbp = ufob.FBP(bp_props={"axis_pos": W / 2.0, "compensated": compensated}, storage=storage)
    vol = fbp.process(stack)
    torch.cuda.synchronize()
    ufob.device_status()
    got = np.stack([vol[i, ry:ry + side, rx:rx + side].double().cpu().numpy() for i in picks])
    assert oracle.rel_l2(got, np.stack(refs)) < tol


@pytest.mark.skipif(not reference.available(), reason="the reference's CPU build (oracle/_ref) is absent")
def test_c1_group_plain_vs_reference(c1_group):
    stack, picks, (rx, ry, side), host, refs = c1_group
    W = stack.shape[-1]
    vol = ufob.FBP(bp_props={"axis_pos": W / 2.0}).process(stack)
    got = np.stack([vol[i, ry:ry + side, rx:rx + side].double().cpu().numpy() for i in picks])
    theirs = np.stack([reference.backproject(reference.fft_filter_ifft(s).astype(np.float32), axis_pos=W / 2.0,
                                             roi_x=rx, roi_y=ry, roi_width=side, roi_height=side) for s in host])
    assert oracle.rel_l2(got, theirs) < 1e-4
    # and the reference build agrees with the FP64 oracle to its own FP32 coordinate and sum
    # rounding (7e-5 measured here, against 1.7e-5 for the engine)
    assert oracle.rel_l2(theirs, np.stack(refs)) < 1e-4


BATCH_SHAPES = [(2048, 1800), (1536, 1750), (256, 180), (1024, 1203), (512, 700), (2048, 997), (256, 1800)]


def busiest_block(img, n):
    """Top-left corner of the n x n block (on an n/2 grid) with the largest energy: a region
    that holds the phantom, not an empty patch whose tiny norm would inflate a relative error."""
    e = torch.nn.functional.avg_pool2d((img * img)[None, None], n, stride=n // 2)[0, 0]
    k = int(torch.argmax(e))
    return (k // e.shape[1]) * (n // 2), (k % e.shape[1]) * (n // 2)


@pytest.fixture(scope="module")
def wide_batch(cuda):
    jobs = []
    for i, (W, P) in enumerate(BATCH_SHAPES):
        sino = oracle.ellipse_sinogram(oracle.random_ellipses(500 + i), W, np.arange(P) * math.pi / P)
        jobs.append(dict(sino=torch.from_numpy(sino.astype(np.float32)).cuda(),
                         out=torch.zeros((W, W), device="cuda")))
    return jobs


# FP32 bound: up to 1800 uncompensated FP32 sums per pixel
@pytest.mark.parametrize("storage,tol", [(ufob.F32, 3e-5), (ufob.F16, 1e-3), (ufob.BF16, 8e-3)])
def test_wide_uneven_batch(wide_batch, storage, tol, tmp_path, monkeypatch):
    monkeypatch.setenv("UFOB_TUNE_CACHE", str(tmp_path / "tune.txt"))
    jobs = wide_batch
    b = ufob.Batch(storage=storage)
    refs = None
    for _ in range(2):  # the first call autotunes, the second replays the captured graph
        for j in jobs:
            j["out"].zero_()
        b.run(jobs)
        torch.cuda.synchronize()
        ufob.device_status()
        if refs is None:  # oracle of each job's graph on a 128^2 region (whole slice up to 256^2)
            refs = []
            for j in jobs:
                W = j["sino"].shape[-1]
                n = W if W <= 256 else 128
                y, x = (0, 0) if W <= 256 else busiest_block(j["out"], n)
                N = 1 << (W - 1).bit_length()
                filt = oracle.fft_filter_ifft(j["sino"].cpu().numpy(), size_x=N, crop_width=W).astype(np.float32)
                refs.append((y, x, n, oracle.backproject(filt, roi_x=x, roi_y=y, roi_width=n, roi_height=n)))
        for j, (y, x, n, ref) in zip(jobs, refs):
            got = j["out"][y:y + n, x:x + n].double().cpu().numpy()
            assert oracle.rel_l2(got, ref) < tol, tuple(j["sino"].shape)


def test_cone_1024_projections(cuda):
    """1024 projections of 512^2 over 360 degrees, source 400 px before the axis and
    detector 100 px behind it (the benchmarked cone geometry at half scale), into 192^3."""
    n, det, vol = 1024, 512, 192
    rng = np.random.default_rng(9)
    proj = rng.uniform(0.0, 1.0, (n, det, det)).astype(np.float32)
    h = vol / 2.0
    props = {"center-position-x": det / 2.0, "center-position-z": det / 2.0,
             "source-position-y": -400.0, "detector-position-y": 100.0}
    t = ufob.GeneralBackprojectTask(num_projections=n)
    for k, v in props.items():
        t.set_property(k, v)
    t.set_property("x-region", (-h, h, 1.0))
    t.set_property("y-region", (-h, h, 1.0))
    t.set_property("region", (-h, h, 1.0))
    got = t.process(torch.from_numpy(proj).cuda())
    torch.cuda.synchronize()
    ufob.device_status()
    assert tuple(got.shape) == (vol, vol, vol)
    for iz in (3, vol // 2, vol - 20):
        z = -h + iz
        ref = oracle.general_backproject(proj, n, region=(z, z + 1.0, 1.0), x_region=(-h, h, 1.0),
                                         y_region=(-h, h, 1.0), **props)[0]
        assert oracle.rel_l2(got[iz].double().cpu().numpy(), ref) < 1e-4, iz
