"""Case lists shared by the golden-fixture tests (must match tests/golden/make_golden.py)."""
import os

import numpy as np

FILTER_CASES = [
    dict(filter="ramp-fromreal"), dict(filter="ramp"), dict(filter="butterworth", cutoff=0.3, order=6.0),
    dict(filter="faris-byer", tau=0.2, theta=0.7), dict(filter="hamming", cutoff=0.4), dict(filter="bh3"),
    dict(filter="ramp-fromreal", scale=1.7), dict(filter="butterworth", scale=0.5),
]
CHAIN_CASES = [dict(), dict(size_x=128, crop_width=100), dict(size_x=128), dict(filter="hamming", cutoff=0.4),
               dict(filter="ramp")]
BP_CASES = [dict(), dict(axis_pos=31.5), dict(axis_pos=30.25, angle_step=0.05, angle_offset=0.3),
            dict(roi_x=10, roi_y=5, roi_width=40, roi_height=30), dict(num_projections=80, offset=20),
            dict(mode="nearest", roi_x=3, roi_width=50, roi_height=50)]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fbp.npz")


def load():
    return dict(np.load(GOLDEN))


def nearest_agrees(got, ref, frac=0.995):
    """mode=nearest truncates the detector coordinate, so rounding-order
    differences flip single taps at exact boundaries; require nearly all
    pixels to agree instead of a norm bound."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    close = np.abs(got - ref) <= 1e-5 * max(np.abs(ref).max(), 1e-30)
    return close.mean() >= frac
