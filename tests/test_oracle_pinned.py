"""The FP64 oracle against the reference itself (CPU, no GPU needed).

Golden fixtures in tests/golden/ were produced by the reference's own task code
and kernels compiled for the CPU (tests/golden/make_golden.py); where that CPU
build is present (oracle/_ref/), the oracle is also compared live on more
seeded cases."""
import math

import numpy as np
import pytest

import golden_cases as gc
import oracle

G = gc.load()


@pytest.mark.parametrize("i", range(len(gc.FILTER_CASES)))
@pytest.mark.parametrize("n", [8, 64, 256])
def test_coefficients_golden(i, n):
    ref = G["coeff_%d_%d" % (i, n)]
    got = oracle.filter_coefficients(n, **gc.FILTER_CASES[i])
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-7 * max(np.abs(ref).max(), 1e-30))


@pytest.mark.parametrize("i", range(len(gc.CHAIN_CASES)))
def test_filter_chain_golden(i):
    got = oracle.fft_filter_ifft(G["chain_input"], **gc.CHAIN_CASES[i])
    assert oracle.rel_l2(got, G["chain_%d" % i]) < 1e-6


@pytest.mark.parametrize("i", range(len(gc.BP_CASES)))
def test_backproject_golden(i):
    c = gc.BP_CASES[i]
    got = oracle.backproject(G["bp_input"], **c)
    ref = G["bp_%d" % i]
    assert got.shape == ref.shape
    if c.get("mode") == "nearest":
        assert gc.nearest_agrees(got, ref)
    else:
        assert oracle.rel_l2(got, ref) < 1e-5


def test_fbp_golden():
    got = oracle.fbp(G["fbp_input"], axis_pos=63.5)
    assert oracle.rel_l2(got, G["fbp_output"]) < 1e-5


def test_forwardproject_golden():
    got = oracle.forwardproject(G["fp_input"], 30, 32.0, math.pi / 30)
    assert oracle.rel_l2(got, G["fp_output"]) < 1e-4


def test_filter_width_error_matches_reference_text():
    with pytest.raises(ValueError, match="must be a power of two"):
        oracle.filter_coefficients(300)


# ------------------------------------------------------------------ live reference (where built)

reference = pytest.importorskip("reference")
live = pytest.mark.skipif(not reference.available(), reason="reference CPU build (oracle/_ref) not present")


@live
@pytest.mark.parametrize("seed", range(6))
def test_live_random_configs(seed):
    rng = np.random.default_rng(100 + seed)
    W = int(rng.choice([32, 64, 128]))
    P = int(rng.integers(8, 90))
    sino = rng.standard_normal((P, W)).astype(np.float32)
    f = dict(filter=str(rng.choice(oracle.FILTERS)), cutoff=float(rng.uniform(0.1, 1.0)),
             scale=float(rng.uniform(0.5, 2.0)))
    size_x = int(rng.choice([0, 2 * W]))
    np.testing.assert_allclose(oracle.fft_filter_ifft(sino, size_x=size_x, **f),
                               reference.fft_filter_ifft(sino, size_x=size_x, **f), rtol=0,
                               atol=1e-5 * np.abs(sino).max() * max(1.0, f["scale"]))
    filt = rng.standard_normal((P, W)).astype(np.float32)
    props = dict(axis_pos=float(rng.uniform(W / 4, 3 * W / 4)), angle_offset=float(rng.uniform(0, 1)),
                 roi_x=int(rng.integers(0, W // 4)), roi_y=int(rng.integers(0, W // 4)),
                 roi_width=int(rng.integers(1, W)), roi_height=int(rng.integers(1, W)))
    assert oracle.rel_l2(oracle.backproject(filt, **props), reference.backproject(filt, **props)) < 1e-5


@live
def test_live_c0_slice():
    """Config 0 at full size: 512 x 512 slice, 512 angles, axis 255.5."""
    ell = oracle.random_ellipses(0)
    s = oracle.ellipse_sinogram(ell, 512, np.arange(512) * math.pi / 512).astype(np.float32)
    assert oracle.rel_l2(oracle.fbp(s, axis_pos=255.5), reference.fbp(s, axis_pos=255.5)) < 1e-5
