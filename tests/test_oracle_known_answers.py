"""Known-answer tests of the oracle itself (no GPU).

The reference pins only its FFT stage with tests; for filter/backproject the
oracle is checked against results that follow from the mathematics: the
analytic Radon pair of an ellipse phantom, a delta sinogram giving a line, a
constant sinogram giving a disc profile, and the half-turn symmetry of the
angle offset (src/ufo-backproject-task.c:174-196: angles = offset + i * step)."""
import math

import numpy as np

import oracle


def test_analytic_radon_pair_ellipses():
    """FBP of the analytic line integrals of ellipses reproduces the ellipses."""
    W, P = 256, 400
    ell = oracle.random_ellipses(3, n=6)
    sino = oracle.ellipse_sinogram(ell, W, np.arange(P) * math.pi / P).astype(np.float32)
    rec = oracle.fbp(sino, axis_pos=W / 2.0, filter_props={"filter": "ramp"})
    img = oracle.ellipse_image(ell, W)
    yy, xx = np.mgrid[0:W, 0:W]
    inner = (xx - W / 2 + 0.5) ** 2 + (yy - W / 2 + 0.5) ** 2 < (0.8 * W / 2) ** 2
    assert oracle.rel_l2(rec[inner], img[inner]) < 0.15


def test_delta_sinogram_gives_a_line():
    """One non-zero bin at angle 0 backprojects to a column: h = bx + axis there."""
    W, P = 64, 8
    sino = np.zeros((P, W), np.float32)
    sino[0, 20] = 1.0
    out = oracle.backproject(sino, axis_pos=W / 2.0)
    # only angle 0 contributes, through bins 20 (and its linear neighbours): a vertical line
    cols = np.nonzero(np.abs(out).sum(axis=0) > 0)[0]
    assert set(cols) <= {19, 20, 21}
    assert np.allclose(out[:, 20], out[0, 20]) and out[0, 20] > 0
    # the column value is the pixel-centre sample times pi / P
    np.testing.assert_allclose(out[0, 20], math.pi / P, rtol=1e-6)


def test_constant_sinogram_gives_disc_profile():
    """A constant sinogram (every ray hits the same value) backprojects to pi * c
    inside the detector's reach (all angles read inside the row)."""
    W, P, c = 64, 180, 0.5
    out = oracle.backproject(np.full((P, W), c, np.float32), axis_pos=W / 2.0)
    yy, xx = np.mgrid[0:W, 0:W]
    r = np.hypot(xx - W / 2 + 0.5, yy - W / 2 + 0.5)
    np.testing.assert_allclose(out[r < W / 2 - 2], math.pi * c, rtol=1e-6)
    assert np.all(out[r > W / 2 * math.sqrt(2) - 0.5] < math.pi * c)


def test_angle_offset_by_pi_is_a_half_turn():
    """Angles shifted by pi flip h about the axis: the image turns by 180 degrees."""
    W, P = 48, 90
    sino = oracle.ellipse_sinogram(oracle.random_ellipses(9), W, np.arange(P) * math.pi / P).astype(np.float32)
    a = oracle.backproject(sino, axis_pos=W / 2.0)
    b = oracle.backproject(sino, axis_pos=W / 2.0, angle_offset=math.pi)
    np.testing.assert_allclose(b, a[::-1, ::-1], rtol=1e-9, atol=1e-9 * np.abs(a).max())


def test_filter_chain_is_linear_and_shift_equivariant():
    """fft ! filter ! ifft is a circular convolution: linear, and a cyclic shift of
    the input shifts the output (no padding by default)."""
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal((2, 3, 128))
    f = oracle.fft_filter_ifft
    np.testing.assert_allclose(f(2 * x - y), 2 * f(x) - f(y), atol=1e-10)
    np.testing.assert_allclose(f(np.roll(x, 5, axis=-1)), np.roll(f(x), 5, axis=-1), atol=1e-10)
