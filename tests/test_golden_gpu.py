"""The CUDA engine against the golden fixtures produced by the reference's own
task code and kernels (tests/golden/make_golden.py)."""
import numpy as np
import pytest
import torch

import golden_cases as gc
import oracle
import ufob

pytestmark = pytest.mark.gpu
G = gc.load()


@pytest.mark.parametrize("i", range(len(gc.FILTER_CASES)))
def test_coefficients(cuda, i):
    for n in (8, 64, 256):
        ref = G["coeff_%d_%d" % (i, n)]
        got = ufob.FilterTask(**gc.FILTER_CASES[i]).coefficients(n)
        np.testing.assert_allclose(got, ref, rtol=0, atol=2e-7 * max(np.abs(ref).max(), 1e-30))


@pytest.mark.parametrize("i", range(len(gc.CHAIN_CASES)))
def test_filter_chain(cuda, i):
    f = ufob.FilterTask(**gc.CHAIN_CASES[i])
    got = f.process(torch.from_numpy(G["chain_input"]).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, G["chain_%d" % i]) < 2e-6


@pytest.mark.parametrize("i", range(len(gc.BP_CASES)))
def test_backproject(cuda, i):
    c = gc.BP_CASES[i]
    got = ufob.BackprojectTask(**c).process(torch.from_numpy(G["bp_input"]).cuda()).cpu().numpy()
    ref = G["bp_%d" % i]
    assert got.shape == ref.shape
    if c.get("mode") == "nearest":
        assert gc.nearest_agrees(got, ref)
    else:
        assert oracle.rel_l2(got, ref) < 1e-5


def test_fbp(cuda):
    got = ufob.FBP(bp_props=dict(axis_pos=63.5)).process(torch.from_numpy(G["fbp_input"]).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, G["fbp_output"]) < 1e-5
