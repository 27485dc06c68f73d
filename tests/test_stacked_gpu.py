"""stacked-backproject on the GPU against the oracle, in its three precision
modes.

Reference: src/ufo-stacked-backproject-task.c:200-430 and
src/kernels/stacked-backproject.cl.  Tolerances: "single" is the FP32
backprojector (≤ 1e-5 relative L2 vs FP64), "half" the FP16 slice-quad
backprojector (≤ 1e-3 vs the oracle on FP16-rounded sinograms), "int8" samples
the nearest texel, where FP32 and FP64 coordinates pick different texels for a
few rays (≤ 2e-3)."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _stack(seed, Z, P, W, filtered=True):
    ang = np.arange(P) * math.pi / P
    s = np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(seed + z), W, ang) for z in range(Z)])
    if filtered:
        s = oracle.fft_filter_ifft(s)
    return s.astype(np.float32)


CASES = [dict(), dict(roi_x=8, roi_y=24, roi_width=48, roi_height=32), dict(axis_pos=61.25, angle_offset=0.3),
         dict(num_projections=200, offset=7, angle_step=math.pi / 210)]
TOL = {"single": 1e-5, "half": 1e-3, "int8": 2e-3}


@pytest.mark.parametrize("mode", ["single", "half", "int8"])
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("Z", [1, 6])
def test_stacked_matches_oracle(cuda, mode, case, Z):
    P, W = 180, 128
    s = _stack(20 + case, Z, P, W)
    props = CASES[case]
    t = ufob.StackedBackprojectTask(precision_mode=mode, **props)
    got = t.process(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = oracle.stacked_backproject(s, mode, **props)
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < TOL[mode], oracle.rel_l2(got, ref)


def test_stacked_single_is_backproject_mirrored(cuda):
    s = torch.from_numpy(_stack(40, 3, 150, 64)).cuda()
    st = ufob.StackedBackprojectTask().process(s)
    bp = ufob.BackprojectTask().process(s)
    assert oracle.rel_l2(st.flip(1).cpu().numpy(), bp.cpu().numpy()) < 1e-6


def test_stacked_int8_dequantisation(cuda):
    """Integer sums and the reference's dequantisation (minimum added once)."""
    P, W = 64, 32
    s = np.full((2, P, W), 3.0, np.float32)
    s[0, 0, 0] = 1.0
    t = ufob.StackedBackprojectTask(precision_mode="int8", roi_x=8, roi_y=8, roi_width=16, roi_height=16)
    got = t.process(torch.from_numpy(s).cuda()).cpu().numpy()
    np.testing.assert_allclose(got, oracle.stacked_backproject(s, "int8", roi_x=8, roi_y=8, roi_width=16,
                                                               roi_height=16), rtol=1e-6)


def test_stacked_many_angles_int8_lane_flush(cuda):
    """More than 256 angles: the 16-bit lane sums are flushed every 256 angles."""
    P, W = 700, 64
    s = np.abs(_stack(50, 4, P, W, filtered=False))
    t = ufob.StackedBackprojectTask(precision_mode="int8")
    got = t.process(torch.from_numpy(s).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, oracle.stacked_backproject(s, "int8")) < 2e-3
