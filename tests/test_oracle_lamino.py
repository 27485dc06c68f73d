"""lamino-backproject oracle and host logic (no GPU).

Reference: src/ufo-lamino-backproject-task.c and the kernels generated from
src/kernels/templates/*_template.in.  The reference ships no test for this
task; the known answer is the tomographic limit: at a laminographic angle of
pi/2 each slice reads one detector row, so the volume is `backproject` of the
sinograms formed by those rows."""
import math

import numpy as np
import pytest

import oracle
import ufob


def _sino_stack(seed, Z, P, W):
    ang = np.arange(P) * math.pi / P
    return np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(seed + z), W, ang) for z in range(Z)])


def tomographic_limit_case(Z=4, P=60, W=48):
    sinos = _sino_stack(7, Z, P, W).astype(np.float32)   # [Z, P, W]
    proj = np.ascontiguousarray(sinos.transpose(1, 0, 2))  # [P, Z, W]: detector row r = slice r
    props = dict(num_projections=P, x_region=(-W // 2, W // 2, 1), y_region=(-W // 2, W // 2, 1),
                 region=(0.0, float(Z), 1.0), center=(W / 2 + 0.5, 0.5), lamino_angle=math.pi / 2)
    return sinos, proj, props


def test_tomographic_limit_is_backproject():
    sinos, proj, props = tomographic_limit_case()
    W = sinos.shape[-1]
    vol = oracle.lamino_backproject(proj, **props)
    ref = oracle.backproject(sinos, axis_pos=W / 2 + 0.5)
    assert vol.shape == ref.shape
    assert oracle.rel_l2(vol, ref) < 1e-5


def test_region_sizes_and_sweeps():
    proj = np.zeros((4, 8, 8), np.float32)
    # REGION_SIZE = (to - from - 1) / step + 1 in integers; nz = ceil((to - from) / step)
    v = oracle.lamino_backproject(proj, 4, (-5, 6, 2), (0, 7, 3), (0.0, 1.0, 0.3))
    assert v.shape == (4, 3, 6)
    for par in ("x-center", "lamino-angle", "roll-angle"):
        assert oracle.lamino_backproject(proj, 4, (0, 4, 1), (0, 4, 1), (0.0, 0.5, 0.1), parameter=par).shape == \
            (5, 4, 4)


def test_lamino_task_properties_and_errors():
    t = ufob.LaminoBackprojectTask()
    with pytest.raises(ufob.UfobError):  # Number of projections has not been set
        t.setup()
    t.set_property("num-projections", 10)
    with pytest.raises(ufob.UfobError):  # Step in region is 0
        t.setup()
    t.set_property("region", (0.0, 4.0, 1.0))
    t.setup()
    t.set_property("x-region", (-8, 8, 1))
    t.set_property("y-region", (-4, 4, 2))
    assert t.get_requisition() == (16, 4, 4)
    t.set_property("x-region", (8, -8, 1))  # from > to: refused with a warning, old value kept
    assert t.get_requisition() == (16, 4, 4)
    t.set_property("parameter", "roll-angle")
    t.set_property("addressing-mode", "clamp_to_edge")
    with pytest.raises(ufob.UfobError):
        t.set_property("parameter", "tilt")
    with pytest.raises(ufob.UfobError):
        t.set_property("addressing-mode", "repeat")
        t.setup()
    assert isinstance(ufob.get_task("lamino-backproject"), ufob.LaminoBackprojectTask)
