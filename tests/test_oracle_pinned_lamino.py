"""The oracle's lamino-backproject against the reference itself (CPU, no GPU needed).

tests/golden/reference_lamino.npz holds the volumes of the reference's own lamino-backproject task
(src/ufo-lamino-backproject-task.c with the kernels src/kernels/tools/make_burst_kernels.py writes
from src/kernels/templates/*_template.in, compiled for the CPU; tests/golden/make_golden.py)."""
import json

import numpy as np
import pytest

import lamino_cases
import oracle

G = lamino_cases.load()
CASES = json.loads(str(G["cases"]))


def test_fixture_matches_case_list():
    assert CASES == json.loads(json.dumps(lamino_cases.CASES))
    np.testing.assert_array_equal(lamino_cases.make_input(), G["input"])


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_lamino(case):
    proj = G["input"]
    ref = G["out_" + case["name"]]
    got = oracle.lamino_backproject(proj, **lamino_cases.oracle_kwargs(case["props"], proj.shape[0]))
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < 1e-5, oracle.rel_l2(got, ref)
