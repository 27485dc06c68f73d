"""Ramp-filter stage (fused fft ! filter ! ifft) against the FP64 oracle.

Reference: src/ufo-filter-task.c:162-336, src/kernels/filter.cl:20-29,
src/ufo-fft-task.c:123-336, src/ufo-ifft-task.c:111-311."""
import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return oracle.rel_l2(a, b)


@pytest.mark.parametrize("filt", oracle.FILTERS)
def test_coefficients_match_reference_builders(cuda, filt):
    f = ufob.FilterTask(filter=filt)
    got = f.coefficients(256)
    ref = oracle.filter_coefficients(256, filter=filt)
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7 * np.abs(ref).max())


@pytest.mark.parametrize("filt", oracle.FILTERS)
@pytest.mark.parametrize("W,H,size_x,crop", [(512, 37, 0, 0), (64, 9, 128, 100), (1024, 4, 0, 1000),
                                             (300, 5, 512, 300), (2048, 3, 0, 0), (8, 1, 0, 0)])
def test_filter_rows_match_oracle(cuda, filt, W, H, size_x, crop):
    rng = np.random.default_rng(W + H)
    sino = rng.standard_normal((H, W)).astype(np.float32)
    f = ufob.FilterTask(filter=filt, size_x=size_x, crop_width=crop)
    got = f.process(torch.from_numpy(sino).cuda()).cpu().numpy()
    ref = oracle.fft_filter_ifft(sino, size_x=size_x, crop_width=crop, filter=filt)
    assert got.shape == ref.shape
    assert _rel(got, ref) < 2e-6


@pytest.mark.parametrize("dtype,tol", [(ufob.F16, 2e-3), (ufob.BF16, 1.5e-2)])
def test_filter_reduced_precision_rows(cuda, dtype, tol):
    rng = np.random.default_rng(1)
    sino = rng.standard_normal((16, 512)).astype(np.float32)
    f = ufob.FilterTask()
    got = f.process(torch.from_numpy(sino).cuda(), dtype=dtype).float().cpu().numpy()
    assert _rel(got, oracle.fft_filter_ifft(sino)) < tol


@pytest.mark.parametrize("dtype", [ufob.F16, ufob.BF16])
def test_filter_pair_layout(cuda, dtype):
    rng = np.random.default_rng(2)
    W = 250
    sino = rng.standard_normal((5, W)).astype(np.float32)
    f = ufob.FilterTask(size_x=256, crop_width=W)
    pairs = f.process(torch.from_numpy(sino).cuda(), dtype=dtype, layout=ufob.PAIRS)
    assert pairs.shape == (5, (W + 1 + 3) // 4 * 4)
    tdt = torch.float16 if dtype == ufob.F16 else torch.bfloat16
    halves = pairs.cpu().view(tdt).float().numpy().reshape(5, -1, 2)
    ref = oracle.fft_filter_ifft(sino, size_x=256, crop_width=W)
    lo, hi = halves[:, :, 0], halves[:, :, 1]
    # pair j = (s[j-1], s[j]) with zeros outside [0, W)
    tol = 2e-3 if dtype == ufob.F16 else 1.5e-2
    assert _rel(hi[:, :W], ref) < tol
    assert _rel(lo[:, 1:W + 1], ref) < tol
    assert np.all(lo[:, 0] == 0) and np.all(hi[:, W:] == 0) and np.all(lo[:, W + 1:] == 0)


def test_filter_spectrum_only(cuda):
    """The reference `filter` task alone multiplies the interleaved spectrum."""
    rng = np.random.default_rng(3)
    spec = rng.standard_normal((7, 2 * 128)).astype(np.float32)
    f = ufob.FilterTask(filter="hamming", cutoff=0.3)
    got = f.apply_spectrum(torch.from_numpy(spec).cuda()).cpu().numpy()
    c = oracle.filter_coefficients(128, filter="hamming", cutoff=0.3).astype(np.float32)
    np.testing.assert_allclose(got, spec * c[None, :], rtol=1e-6)


def test_filter_linearity_and_zero(cuda):
    rng = np.random.default_rng(4)
    a = torch.from_numpy(rng.standard_normal((8, 1024)).astype(np.float32)).cuda()
    b = torch.from_numpy(rng.standard_normal((8, 1024)).astype(np.float32)).cuda()
    f = ufob.FilterTask()
    fa, fb, fab = f.process(a), f.process(b), f.process(2 * a - 3 * b)
    assert _rel((fab).cpu().numpy(), (2 * fa - 3 * fb).cpu().numpy()) < 1e-5
    assert torch.count_nonzero(f.process(torch.zeros_like(a))) == 0
