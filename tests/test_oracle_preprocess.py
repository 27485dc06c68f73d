"""Oracle and host logic of the preprocessing tasks (no GPU).

Reference: src/kernels/ffc.cl:20-50, src/ufo-flat-field-correct-task.c,
src/ufo-transpose-projections-task.c:60-120,
src/ufo-cone-beam-projection-weight-task.c:113-151, src/kernels/conebeam.cl:20-36.
The reference ships no tests for these tasks; the known answers below follow
from the kernels' formulas."""
import math

import numpy as np
import pytest

import oracle
import ufob


def _frames(seed, n, H, W):
    rng = np.random.default_rng(seed)
    dark = rng.uniform(90, 110, (H, W)).astype(np.float32)
    flat = (dark + rng.uniform(800, 1200, (H, W))).astype(np.float32)
    data = (dark + rng.uniform(50, 1000, (n, H, W))).astype(np.float32)
    return data, dark, flat


def test_ffc_known_answers():
    data, dark, flat = _frames(1, 2, 5, 7)
    # data == flat -> 1, data == dark -> 0; absorption: log(1) = 0 and log(x/0) = inf
    np.testing.assert_array_equal(oracle.flat_field_correct(flat[None], dark, flat)[0], np.ones_like(flat))
    np.testing.assert_array_equal(oracle.flat_field_correct(dark[None], dark, flat)[0], np.zeros_like(flat))
    assert np.all(oracle.flat_field_correct(flat, dark, flat, absorption_correct=True) == 0)
    r = oracle.flat_field_correct(dark, dark, flat, absorption_correct=True)
    assert np.all(np.isinf(r))
    assert np.all(oracle.flat_field_correct(dark, dark, flat, absorption_correct=True, fix_nan_and_inf=True) == 0)
    # absorption = -log(transmission)
    t = oracle.flat_field_correct(data, dark, flat)
    a = oracle.flat_field_correct(data, dark, flat, absorption_correct=True)
    np.testing.assert_allclose(a, -np.log(t.astype(np.float64)), rtol=1e-5, atol=1e-6)


def test_ffc_scales_and_sinogram_input():
    data, dark, flat = _frames(2, 1, 4, 9)
    r = oracle.flat_field_correct(data, dark, flat, dark_scale=0.5, flat_scale=2.0)
    ref = (data - dark * 0.5) / (flat * 2.0 - dark * 0.5)
    np.testing.assert_allclose(r, ref, rtol=2e-7)
    # sinogram input: one dark/flat row for every row
    r = oracle.flat_field_correct(data[0], dark[0], flat[0], sinogram_input=True)
    np.testing.assert_allclose(r, (data[0] - dark[0]) / (flat[0] - dark[0]), rtol=2e-7)


def test_transpose_round_trip():
    p = np.arange(3 * 4 * 5, dtype=np.float32).reshape(3, 4, 5)
    s = oracle.transpose_projections(p)
    assert s.shape == (4, 3, 5)
    for y in range(4):
        for i in range(3):
            np.testing.assert_array_equal(s[y, i], p[i, y])
    np.testing.assert_array_equal(oracle.transpose_projections(s), p)


def test_cone_weight_known_answers():
    sd, dd = 300.0, 100.0
    H, W = 6, 8
    ones = np.ones((H, W), np.float32)
    # tomography (cos = 1): overall distance = source distance, so the pixel whose
    # magnified offset is 0 gets sd / sd = 1 and others sd / sqrt(sd^2 + r^2)
    w = oracle.cone_beam_weight(ones, center_position_x=W / 2 - 0.5 + 0.0, center_position_z=H / 2 - 0.5,
                                source_distance=sd, detector_distance=dd)
    cx, cz = W / 2 - 0.5, H / 2 - 0.5
    mr = sd / (sd + dd)
    for y in range(H):
        for x in range(W):
            u, v = (x - cx + 0.5) * mr, (y - cz + 0.5) * mr
            np.testing.assert_allclose(w[y, x], sd / math.sqrt(sd * sd + u * u + v * v), rtol=1e-6)
    # laminography: cos(angle) scales the weight and the overall distance is sd + dd
    ang = 0.4
    w2 = oracle.cone_beam_weight(ones, center_position_x=cx, center_position_z=cz, source_distance=sd,
                                 detector_distance=dd, axis_angle_x=ang)
    u, v = (0 - cx + 0.5) * mr, (0 - cz + 0.5) * mr
    np.testing.assert_allclose(w2[0, 0], sd * math.cos(ang) / math.sqrt((sd + dd) ** 2 + u * u + v * v), rtol=1e-6)


def test_cone_weight_per_projection_values():
    ones = np.ones((3, 2, 4), np.float32)
    w = oracle.cone_beam_weight(ones, center_position_x=[1.0, 2.0, 3.0], center_position_z=1.0,
                                source_distance=[100.0, 200.0, 300.0], detector_distance=10.0)
    for i in range(3):
        ref = oracle.cone_beam_weight(ones[i], center_position_x=1.0 + i, center_position_z=1.0,
                                      source_distance=100.0 * (i + 1), detector_distance=10.0)
        np.testing.assert_array_equal(w[i], ref)
    # a later call starts at its first index
    np.testing.assert_array_equal(
        oracle.cone_beam_weight(ones[:1], first=2, center_position_x=[1.0, 2.0, 3.0], center_position_z=1.0,
                                source_distance=[100.0, 200.0, 300.0], detector_distance=10.0)[0], w[2])
    with pytest.raises(IndexError):  # the reference asserts on a missing value
        oracle.cone_beam_weight(ones, center_position_x=[1.0, 2.0], center_position_z=1.0, source_distance=1.0,
                                detector_distance=1.0)


def test_ffc_props_defaults_and_names():
    t = ufob.FlatFieldCorrectTask()
    assert t.get_property("fix-nan-and-inf") is False
    assert t.get_property("absorption-correct") is False
    assert t.get_property("sinogram-input") is False
    assert t.get_property("dark-scale") == 1.0 and t.get_property("flat-scale") == 1.0
    t.set_property("absorption-correct", True)
    t.set_property("dark_scale", 0.25)
    assert t.get_property("absorption-correct") is True and t.get_property("dark-scale") == 0.25
    with pytest.raises(ufob.UfobError):
        t.set_property("gain", 2.0)


def test_cone_weight_handle_properties():
    w = ufob.ConeBeamProjectionWeightTask(source_distance=100.0)
    w.set_property("center-position-x", [1.0, 2.0])
    w.set_property("axis-angle-x", 0.0)
    assert w.count == 0
    w.count = 5
    assert w.count == 5
    with pytest.raises(ufob.UfobError):
        w.set_property("detector-position-y", 1.0)


def test_task_table_names():
    assert isinstance(ufob.get_task("flat-field-correct"), ufob.FlatFieldCorrectTask)
    assert isinstance(ufob.get_task("cone-beam-projection-weight"), ufob.ConeBeamProjectionWeightTask)
    t = ufob.get_task("transpose-projections", num_projections=12)
    assert t.get_requisition(64, 32) == (64, 12)
    with pytest.raises(ufob.UfobError):
        t.set_property("offset", 1)


# --------------------------------------------------------------------------- stacked-backproject

def _sino_stack(seed, Z, P, W):
    ang = np.arange(P) * math.pi / P
    return np.stack([oracle.ellipse_sinogram(oracle.random_ellipses(seed + z), W, ang) for z in range(Z)])


def test_stacked_orientation_is_backproject_flipped():
    """h = bx cos - by sin + axis: with the default axis W/2 and a full ROI the
    stacked image is the backproject image mirrored in y (by -> -by)."""
    s = _sino_stack(3, 2, 60, 48)
    st = oracle.stacked_backproject(s, "single")
    bp = oracle.backproject(s)
    np.testing.assert_allclose(st, bp[:, ::-1, :], rtol=1e-9, atol=1e-9 * np.abs(bp).max())


def test_stacked_half_and_int8_modes():
    s = _sino_stack(4, 3, 90, 64)
    single = oracle.stacked_backproject(s, "single")
    half = oracle.stacked_backproject(s, "half")
    assert oracle.rel_l2(half, single) < 1e-3
    # int8 on a sinogram whose minimum is 0: the reference's once-added minimum vanishes and the
    # result is a nearest-neighbour backprojection of 8-bit data (compared inside the inscribed
    # circle: outside it rays leave the detector, where int8 clamps to the edge and the others read 0)
    pos = np.maximum(s, 0).astype(np.float32)
    pos[0, 0, 0] = 0.0
    roi = dict(roi_x=16, roi_y=16, roi_width=32, roi_height=32)
    q = oracle.stacked_backproject(pos, "int8", **roi)
    assert oracle.rel_l2(q, oracle.stacked_backproject(pos, "single", **roi)) < 0.02
    with pytest.raises(ValueError):
        oracle.stacked_backproject(s, "double")


def test_stacked_int8_dequantisation_formula():
    """uninterleave_uint adds the minimum once, not once per projection."""
    P, W = 8, 16
    s = np.full((1, P, W), 3.0, np.float32)
    s[0, 0, 0] = 1.0  # min 1, max 3
    out = oracle.stacked_backproject(s, "int8", roi_x=4, roi_y=4, roi_width=4, roi_height=4)
    # every sample away from column 0 quantises to 255 -> sum = 255 P
    expect = (np.float32(255 * P) * np.float32(2.0 / 255.0) + np.float32(1.0)) * np.float32(math.pi) / np.float32(P)
    np.testing.assert_allclose(out, expect, rtol=1e-6)


def test_stacked_task_properties():
    t = ufob.StackedBackprojectTask(precision_mode="half", axis_pos=10.5)
    t.set_property("precision-mode", "int8")
    t.set_property("roi-width", 32)
    assert t.get_requisition(64, 90) == (32, 64)
    with pytest.raises(ufob.UfobError):
        t.set_property("precision-mode", "double")
    with pytest.raises(ufob.UfobError):
        t.set_property("mode", "nearest")
    with pytest.raises(ufob.UfobError):  # more rows than num-projections
        t.set_property("num-projections", 10)
        t.get_requisition(64, 90)
