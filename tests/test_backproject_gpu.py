"""Parallel-beam backprojection against the FP64 oracle.

Reference: src/kernels/backproject.cl:24-94, src/ufo-backproject-task.c:96-267.
Bar: relative L2 <= 1e-5 against the oracle with exact interpolation weights
(FP32 CUDA vs FP64), plain FP32 storage."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _sino(P, W, seed=0, nz=None):
    rng = np.random.default_rng(seed)
    shape = (P, W) if nz is None else (nz, P, W)
    return rng.standard_normal(shape).astype(np.float32)


@pytest.mark.parametrize("P,W", [(512, 512), (90, 512), (37, 100), (1, 64), (180, 257)])
def test_single_slice(cuda, P, W):
    s = _sino(P, W)
    bp = ufob.BackprojectTask()
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = oracle.backproject(s)
    assert got.shape == ref.shape == (W, W)
    assert oracle.rel_l2(got, ref) < 1e-5


@pytest.mark.parametrize("props", [
    dict(axis_pos=255.5), dict(axis_pos=200.25), dict(angle_step=0.01, angle_offset=0.5),
    dict(roi_x=100, roi_y=30, roi_width=200, roi_height=150), dict(num_projections=400, offset=100),
    dict(num_projections=300), dict(roi_width=700, roi_height=600, axis_pos=300.0),
])
def test_properties(cuda, props):
    s = _sino(200, 512, seed=1)
    bp = ufob.BackprojectTask(**props)
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = oracle.backproject(s, **props)
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < 1e-5


@pytest.mark.parametrize("nz", [2, 3, 4, 5, 8, 13])
def test_stack(cuda, nz):
    s = _sino(100, 128, seed=2, nz=nz)
    bp = ufob.BackprojectTask()
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = oracle.backproject(s)
    assert oracle.rel_l2(got, ref) < 1e-5
    for z in range(nz):  # every slice independently right
        assert oracle.rel_l2(got[z], ref[z]) < 1e-5


@pytest.mark.parametrize("tile", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9])
def test_tiles(cuda, tile):
    s = _sino(77, 200, seed=3, nz=9)
    bp = ufob.BackprojectTask(tile=tile, roi_width=150, roi_height=170)
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, oracle.backproject(s, roi_width=150, roi_height=170)) < 1e-5


def test_unaligned_width_restaged(cuda):
    s = _sino(64, 101, seed=4)  # 101 floats per row: not a 16-byte pitch
    bp = ufob.BackprojectTask()
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, oracle.backproject(s)) < 1e-5


def test_nearest_mode(cuda):
    s = _sino(60, 64, seed=5)
    bp = ufob.BackprojectTask(mode="nearest")
    got = bp.process(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = oracle.backproject(s, mode="nearest")
    assert oracle.rel_l2(got, ref) < 1e-4


def test_angle_offset_pi_mirrors(cuda):
    """Known answer: adding pi to every angle maps (x, y) -> (-x, -y) about the axis."""
    W = 128
    s = _sino(90, W, seed=6)
    a = ufob.BackprojectTask(axis_pos=W / 2).process(torch.from_numpy(s).cuda()).cpu().numpy()
    b = ufob.BackprojectTask(axis_pos=W / 2, angle_offset=math.pi).process(
        torch.from_numpy(s).cuda()).cpu().numpy()
    assert oracle.rel_l2(b, a[::-1, ::-1]) < 1e-5


def test_constant_sinogram_gives_disc(cuda):
    """Known answer: a constant sinogram c backprojects to pi*c inside the
    inscribed circle (every ray of every angle hits the detector)."""
    W, P = 256, 180
    s = np.full((P, W), 2.0, dtype=np.float32)
    got = ufob.BackprojectTask().process(torch.from_numpy(s).cuda()).cpu().numpy()
    yy, xx = np.mgrid[:W, :W]
    r = np.hypot(xx + 0.5 - W / 2, yy + 0.5 - W / 2)
    inside = r < W / 2 - 2
    np.testing.assert_allclose(got[inside], 2.0 * math.pi, rtol=2e-6)


@pytest.mark.parametrize("dtype,tol", [(ufob.F16, 1e-3), (ufob.BF16, 8e-3)])
@pytest.mark.parametrize("kahan", [0, 1])
def test_pairs_storage(cuda, dtype, tol, kahan):
    rng = np.random.default_rng(7)
    W, P, nz = 256, 300, 5
    raw = rng.standard_normal((nz, P, W)).astype(np.float32)
    f = ufob.FilterTask()
    pairs = f.process(torch.from_numpy(raw).cuda(), dtype=dtype, layout=ufob.PAIRS)
    bp = ufob.BackprojectTask(compensated=kahan)
    got = bp.process(pairs, dtype=dtype, layout=ufob.PAIRS, width=W).cpu().numpy()
    ref = oracle.backproject(oracle.fft_filter_ifft(raw).astype(np.float32))
    assert oracle.rel_l2(got, ref) < tol


@pytest.mark.parametrize("dtype,tol", [(ufob.F16, 1e-3), (ufob.BF16, 8e-3)])
@pytest.mark.parametrize("tile", [0, 8, 9])
@pytest.mark.parametrize("kahan", [0, 1])
def test_pairs_single_slice_tiles(cuda, dtype, tol, tile, kahan):
    """One 16-bit pair sinogram through the single-slice tiles (32x16, 32x96, 32x32 pixels),
    whose coordinate chain and weight pairs run two output rows at a time."""
    rng = np.random.default_rng(11)
    W, P = 320, 250
    raw = rng.standard_normal((P, W)).astype(np.float32)
    f = ufob.FilterTask(size_x=512, crop_width=W)
    pairs = f.process(torch.from_numpy(raw).cuda(), dtype=dtype, layout=ufob.PAIRS)
    bp = ufob.BackprojectTask(tile=tile, compensated=kahan, roi_width=300, roi_height=290)
    got = bp.process(pairs, dtype=dtype, layout=ufob.PAIRS, width=W).cpu().numpy()
    ref = oracle.backproject(oracle.fft_filter_ifft(raw, size_x=512, crop_width=W).astype(np.float32),
                             roi_width=300, roi_height=290)
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < tol



@pytest.mark.parametrize("dtype,tol", [(ufob.F32, 3e-5), (ufob.F16, 1e-3), (ufob.BF16, 8e-3)])
@pytest.mark.parametrize("groups,tile", [(2, 10), (4, 8), (8, 11), (4, 9), (2, 0)])
def test_single_sinogram_angle_groups(cuda, dtype, tol, groups, tile):
    """A sinogram with 1536 angles backprojected as equal angle groups (the slices of one launch,
    partial images summed in group order; compensated sums for the 16-bit forms), for every
    single-slice tile shape: same result as the oracle and, within round-off, as one launch of the
    same tile.  FP32 bound: 1536 angles of a noise sinogram, whose slice is small against its
    terms."""
    rng = np.random.default_rng(21)
    W, P = 512, 1536
    raw = rng.standard_normal((P, W)).astype(np.float32)
    f = ufob.FilterTask()
    ref = oracle.backproject(oracle.fft_filter_ifft(raw).astype(np.float32))
    if dtype == ufob.F32:
        src, kw = f.process(torch.from_numpy(raw).cuda()), {}
    else:
        src = f.process(torch.from_numpy(raw).cuda(), dtype=dtype, layout=ufob.PAIRS)
        kw = dict(dtype=dtype, layout=ufob.PAIRS, width=W)
    torch.cuda.synchronize()
    n0 = ufob.launch_count()
    got = ufob.BackprojectTask(tile=tile, angle_groups=groups).process(src, **kw).cpu().numpy()
    n1 = ufob.launch_count()
    unsplit = ufob.BackprojectTask(tile=tile, angle_groups=1).process(src, **kw).cpu().numpy()
    n2 = ufob.launch_count()
    # the split run adds exactly one launch: the ordered sum of the partial images
    assert (n1 - n0) == (n2 - n1) + 1
    assert oracle.rel_l2(got, ref) < tol
    assert oracle.rel_l2(got, unsplit) < 1e-5


def test_automatic_plan_matches_oracle(cuda):
    """The automatic tile / angle-group plan of one sinogram at several sizes (whatever it picks)
    against the oracle, and an impossible pinned split is refused."""
    rng = np.random.default_rng(22)
    for W, P in [(512, 512), (256, 256), (1024, 1024), (300, 96), (128, 40)]:
        raw = rng.standard_normal((P, W)).astype(np.float32)
        filt = ufob.FilterTask(size_x=1 << (W - 1).bit_length(), crop_width=W).process(torch.from_numpy(raw).cuda())
        got = ufob.BackprojectTask().process(filt).cpu().numpy()
        ref = oracle.backproject(oracle.fft_filter_ifft(raw, size_x=1 << (W - 1).bit_length(),
                                                        crop_width=W).astype(np.float32))
        assert oracle.rel_l2(got, ref) < 3e-5, (W, P)
    with pytest.raises(ufob.UfobError):
        ufob.BackprojectTask(angle_groups=8).process(filt)  # 40 rows: groups of 5
