"""The CUDA engine's stacked-backproject against the reference's own task in its three precision
modes (tests/golden/reference_stacked.npz, tests/golden/make_golden.py; the reference's kernels
src/kernels/stacked-backproject.cl compiled for the CPU).  "half" stores FP16 texels in the
reference and FP16 slice-quad cells in the engine; "int8" samples the nearest texel, where FP32
coordinates computed in a different order pick the other texel for a few rays."""
import json

import pytest
import torch

import oracle
import stacked_cases
import ufob

pytestmark = pytest.mark.gpu
G = stacked_cases.load()
CASES = json.loads(str(G["cases"]))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_engine_matches_reference_stacked(cuda, case):
    kw = stacked_cases.kwargs(case["props"])
    t = ufob.StackedBackprojectTask(**kw)
    got = t.process(torch.from_numpy(G["input"]).cuda()).cpu().numpy()
    ref = G["out_" + case["name"]]
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < stacked_cases.TOL[kw["precision_mode"]], oracle.rel_l2(got, ref)
