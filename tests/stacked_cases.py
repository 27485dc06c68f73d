"""Cases of the stacked-backproject golden fixtures (tests/golden/reference_stacked.npz).

The reference task (src/ufo-stacked-backproject-task.c:296-430) reconstructs pairs (single) or
quads (half, int8) of slices per image-array texel in 16x16 work-groups; its result is defined for
stacks whose depth is a multiple of the group size and square ROIs whose side is a multiple of 16
(other shapes leave slices unwritten or overlap rows, which the engine does not reproduce).  The
cases stay inside that domain: every precision mode with the default ROI, a shifted axis and angle
offset, an ROI, and a partial sinogram (offset into more num-projections)."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_stacked.npz")
Z, P, W = 4, 90, 48


def make_input(oracle):
    """Filtered sinograms of random-ellipse phantoms [Z, P, W] (the oracle's FP64 ramp filter)."""
    ang = np.arange(P) * math.pi / P
    s = np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(20 + z), W, ang) for z in range(Z)])
    return oracle.fft_filter_ifft(s, size_x=64, crop_width=W).astype(np.float32)


PROPS = [{}, {"axis-pos": 23.25, "angle-offset": 0.3}, {"roi-x": 8, "roi-y": 12, "roi-width": 32, "roi-height": 32},
         {"num-projections": 100, "offset": 7, "angle-step": math.pi / 105}]
CASES = [dict(name="%s_%d" % (mode, i), props=dict(p, **{"precision-mode": mode}))
         for mode in ("single", "half", "int8") for i, p in enumerate(PROPS)]
TOL = {"single": 1e-5, "half": 1e-3, "int8": 2e-3}


def kwargs(props):
    """The oracle's / engine's keyword form of a property set."""
    return {k.replace("-", "_"): v for k, v in props.items()}


def load():
    return dict(np.load(GOLDEN))
