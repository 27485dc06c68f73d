"""The preprocessing oracles against the reference's own kernels (CPU).

tests/golden/reference_pre.npz holds the outputs of src/kernels/ffc.cl and
src/kernels/conebeam.cl compiled for the CPU (oracle/ref.mk,
tests/golden/make_golden.py) on seeded frames; the cone-beam kernel arguments
come from the task's host arithmetic as oracle.cone_weight_params restates it
(src/ufo-cone-beam-projection-weight-task.c:128-139)."""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_pre.npz"))
FFC_CASES = [dict(), dict(absorption_correct=True), dict(absorption_correct=True, fix_nan_and_inf=True),
             dict(dark_scale=0.5, flat_scale=1.5)]
CONE_CASES = [dict(center_position_x=20.5, center_position_z=9.0, source_distance=300.0, detector_distance=100.0),
              dict(center_position_x=17.25, center_position_z=11.5, source_distance=150.0, detector_distance=60.0,
                   axis_angle_x=0.4)]


@pytest.mark.parametrize("i", range(len(FFC_CASES)))
def test_ffc_oracle_matches_reference_kernel(i):
    ref = G["ffc_%d" % i]
    got = oracle.flat_field_correct(G["ffc_data"], G["ffc_dark"], G["ffc_flat"], **FFC_CASES[i])
    fin = np.isfinite(ref)
    np.testing.assert_array_equal(np.isfinite(got), fin)
    # the kernel's float log and the C++ build's FMA contraction differ from NumPy by an ulp or two
    np.testing.assert_allclose(got[fin], ref[fin], rtol=3e-7, atol=1e-7)


@pytest.mark.parametrize("i", range(len(CONE_CASES)))
def test_cone_weight_oracle_matches_reference_kernel(i):
    got = oracle.cone_beam_weight(G["cone_input"], **CONE_CASES[i])
    np.testing.assert_allclose(got, G["cone_%d" % i], rtol=3e-7, atol=1e-7)
