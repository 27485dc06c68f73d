"""The oracle's stacked-backproject against the reference itself (CPU, no GPU needed).

tests/golden/reference_stacked.npz holds the volumes of the reference's own stacked-backproject
task (src/ufo-stacked-backproject-task.c with src/kernels/stacked-backproject.cl compiled for the
CPU, work-groups run as OpenMP teams; tests/golden/make_golden.py) in its three precision modes."""
import json

import numpy as np
import pytest

import oracle
import stacked_cases

G = stacked_cases.load()
CASES = json.loads(str(G["cases"]))


def test_fixture_matches_case_list():
    assert CASES == json.loads(json.dumps(stacked_cases.CASES))
    np.testing.assert_allclose(stacked_cases.make_input(oracle), G["input"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_stacked(case):
    kw = stacked_cases.kwargs(case["props"])
    mode = kw.pop("precision_mode")
    got = oracle.stacked_backproject(G["input"], mode, **kw)
    ref = G["out_" + case["name"]]
    assert got.shape == ref.shape
    # single and half sample with exact weights in both; int8 picks texels by floor(h) in FP32
    assert oracle.rel_l2(got, ref) < {"single": 2e-6, "half": 2e-6, "int8": 1e-4}[mode]
