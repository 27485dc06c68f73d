"""Slice-quad FP16 storage: the filter stage's cell layout and the
backprojection over it (every accumulation mode, Kahan on/off, slice counts
that do not fill the last group of four) against the FP64 oracle."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _raw(nz, P, W, seed):
    return np.random.default_rng(seed).standard_normal((nz, P, W)).astype(np.float32)


# every FFT size of the register-radix filter: its teams meet as half warps (256), on named
# barriers (512, 1024), or as the whole CTA (2048), and one team fills a CTA alone (4096)
@pytest.mark.parametrize("W,N", [(250, 256), (500, 512), (1000, 1024), (2000, 2048), (4000, 4096)])
@pytest.mark.parametrize("nz", [1, 4, 6])
def test_filter_quad_cells(cuda, nz, W, N):
    P = 7
    raw = _raw(nz, P, W, 3)
    f = ufob.FilterTask(size_x=N, crop_width=W)
    q = f.process(torch.from_numpy(raw).cuda(), dtype=ufob.F16, layout=ufob.QUADS)
    G = (nz + 3) // 4
    assert q.shape == (G, P, W + 1, 4)
    h = q.cpu().view(torch.int32).numpy().view(np.float16).astype(np.float32).reshape(G, P, W + 1, 8)
    ref = oracle.fft_filter_ifft(raw.reshape(-1, W), size_x=N, crop_width=W).reshape(nz, P, W)
    for z in range(4 * G):
        g, k = divmod(z, 4)
        lo, hi = h[g, :, :, k], h[g, :, :, 4 + k]
        if z >= nz:
            assert np.all(lo == 0) and np.all(hi == 0)
            continue
        # cell j = (s[j-1], s[j]) per slice, zero outside [0, W)
        assert oracle.rel_l2(hi[:, :W], ref[z]) < 2e-3
        assert oracle.rel_l2(lo[:, 1:], ref[z]) < 2e-3
        assert np.all(lo[:, 0] == 0) and np.all(hi[:, W] == 0)
        # the halves are the FP16 rounding of the rows form: the FFT pairs other rows, so the FP32
        # round-off of the two transforms (growing with N) may move a value by one FP16 step, which
        # for small values is one step of the row's largest value
        rows = f.process(torch.from_numpy(raw[z]).cuda(), dtype=ufob.F16).float().cpu().numpy()
        scale = float(np.abs(rows).max())
        assert np.all(np.abs(hi[:, :W] - rows) <= 2.0 ** -10 * np.abs(rows) + 2.0 ** -11 * scale)
        assert np.mean(hi[:, :W] == rows) > 0.9


@pytest.mark.parametrize("half_sums,tol", [(0, 1e-3), (1, 2e-3)])
@pytest.mark.parametrize("kahan", [0, 1])
@pytest.mark.parametrize("nz", [3, 8, 13])
def test_quads_backprojection(cuda, half_sums, tol, kahan, nz):
    W, P = 256, 300
    raw = _raw(nz, P, W, 11 + nz)
    f = ufob.FilterTask()
    q = f.process(torch.from_numpy(raw).cuda(), dtype=ufob.F16, layout=ufob.QUADS)
    bp = ufob.BackprojectTask(compensated=kahan, half_sums=half_sums)
    got = bp.process(q, layout=ufob.QUADS, width=W, nslices=nz).cpu().numpy()
    ref = oracle.backproject(oracle.fft_filter_ifft(raw.reshape(-1, W)).reshape(nz, P, W).astype(np.float32))
    assert got.shape == (nz, W, W)
    for z in range(nz):
        assert oracle.rel_l2(got[z], ref[z]) < tol, z


@pytest.mark.parametrize("tile", list(range(13)) + [16, 19])
def test_quads_tiles(cuda, tile):
    W, P, nz = 200, 180, 8
    raw = _raw(nz, P, W, 5)
    q = ufob.FilterTask(size_x=256, crop_width=W).process(torch.from_numpy(raw).cuda(), dtype=ufob.F16,
                                                           layout=ufob.QUADS)
    bp = ufob.BackprojectTask(tile=tile, axis_pos=97.25, angle_step=math.pi / 200, roi_x=10, roi_y=20,
                              roi_width=150, roi_height=120)
    got = bp.process(q, layout=ufob.QUADS, width=W, nslices=nz).cpu().numpy()
    filt = oracle.fft_filter_ifft(raw.reshape(-1, W), size_x=256, crop_width=W).reshape(nz, P, W)
    ref = np.stack([oracle.backproject(filt[z].astype(np.float32), axis_pos=97.25, angle_step=math.pi / 200,
                                       roi_x=10, roi_y=20, roi_width=150, roi_height=120) for z in range(nz)])
    assert oracle.rel_l2(got, ref) < 1e-3


def test_fbp_f16_uses_quads_and_matches(cuda):
    nz, P, W = 6, 512, 512
    stack = np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(40 + z), W, np.arange(P) * math.pi / P)
                      for z in range(nz)]).astype(np.float32)
    ref = oracle.fbp(stack)
    for half_sums, tol in ((0, 5e-4), (1, 1e-3)):
        fbp = ufob.FBP(storage=ufob.F16, bp_props={"half_sums": half_sums})
        got = fbp.process(torch.from_numpy(stack).cuda()).cpu().numpy()
        assert oracle.rel_l2(got, ref) < tol, half_sums


def test_quads_layout_rejections(cuda):
    bp = ufob.BackprojectTask()
    q = torch.zeros((1, 10, 65, 4), dtype=torch.int32, device="cuda")
    out = torch.empty((1, 64, 64), device="cuda")
    for dtype in (ufob.F32, ufob.BF16):  # the QUADS layout is F16 only
        with pytest.raises(ufob.UfobError):
            ufob.check(ufob.lib().ufob_backproject_run(bp._h, q.data_ptr(), dtype, ufob.QUADS, 64, 10, 1, 65, 650,
                                                       out.data_ptr(), None))
    with pytest.raises(ufob.UfobError):  # pitch below width + 1 cells
        ufob.check(ufob.lib().ufob_backproject_run(bp._h, q.data_ptr(), ufob.F16, ufob.QUADS, 64, 10, 1, 60, 650,
                                                   out.data_ptr(), None))
    f = ufob.FilterTask()
    with pytest.raises(ufob.UfobError):
        ufob.check(ufob.lib().ufob_filter_run(f._h, q.data_ptr(), 64, 10, 64, q.data_ptr(), ufob.F16, ufob.QUADS,
                                              0, None))
