"""Cases of the lamino-backproject golden fixtures (tests/golden/reference_lamino.npz).

Property sets of the reference task (src/ufo-lamino-backproject-task.c:669-780) over one seeded,
smoothed projection stack: every swept parameter (z, x-center, lamino-angle, roll-angle), a roll
angle, a fixed tomographic angle, clamp_to_edge addressing, a full turn, and a projection count
that leaves a rest for the task's scalar kernel (BURST = 16).  tests/golden/make_golden.py runs
the reference's own task with the kernels its build generates; the oracle (CPU) and the CUDA
engine (GPU) are checked against the stored volumes."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_lamino.npz")
N, H, W = 40, 40, 64  # 40 = 2 bursts of 16 + 8 projections through the scalar kernel


def make_input():
    rng = np.random.default_rng(3)
    p = rng.standard_normal((N, H, W)).astype(np.float32)
    k = np.ones(5, np.float32) / 5  # smooth so that the linear interpolation is well conditioned
    p = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 2, p)
    return np.ascontiguousarray(np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 1, p).astype(np.float32))


BASE = {"x-region": [-24, 24, 1], "y-region": [-20, 28, 2], "center": [W / 2 + 0.25, H / 2 - 1.5],
        "projection-offset": [1, -2], "lamino-angle": 0.6}
CASES = [
    dict(name="z", props=dict(BASE, region=[-6.0, 6.0, 1.5])),
    dict(name="z_roll", props=dict(BASE, region=[-4.0, 4.0, 1.0], **{"roll-angle": 0.12})),
    dict(name="x_center", props=dict(BASE, region=[30.0, 36.0, 1.0], parameter="x-center", z=2.0)),
    dict(name="lamino_sweep", props=dict(BASE, region=[0.3, 0.9, 0.1], parameter="lamino-angle", z=-3.0)),
    dict(name="roll_sweep", props=dict(BASE, region=[-0.2, 0.2, 0.1], parameter="roll-angle", z=1.0)),
    dict(name="tomo_fixed", props=dict(BASE, region=[-2.0, 2.0, 1.0], **{"tomo-angle": 0.4})),
    dict(name="edge", props=dict(BASE, region=[-2.0, 2.0, 1.0], **{"addressing-mode": "clamp_to_edge"})),
    dict(name="overall", props=dict(BASE, region=[-2.0, 2.0, 1.0], **{"overall-angle": 2 * math.pi})),
    dict(name="steep", props=dict(BASE, region=[-3.0, 3.0, 2.0], **{"lamino-angle": 1.2, "x-region": [-30, 31, 3]})),
]


def oracle_kwargs(props, n):
    """The oracle's / engine's keyword form of a property set."""
    kw = {k.replace("-", "_"): (tuple(v) if isinstance(v, list) else v) for k, v in props.items()}
    kw["num_projections"] = n
    return kw


def load():
    return dict(np.load(GOLDEN))
