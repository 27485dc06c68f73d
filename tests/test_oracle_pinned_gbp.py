"""The FP64 oracle's general-backproject against the reference itself (CPU, no GPU needed).

tests/golden/reference_gbp.npz holds the volumes of the reference's own general-backproject task
(src/ufo-general-backproject-task.c with the kernel its make_kernel generates, compiled for the CPU;
tests/golden/make_golden.py) on the cases of tests/gbp_cases.py: every geometry class of the
transform chain (:807-1048), per-projection (vectorised) geometry, every parameter sweep kind,
compute/result/store types with gray mapping, bursts with a rest kernel, chunked volumes, odd sizes
and configuration 2 at reduced size."""
import json

import numpy as np
import pytest

import gbp_cases
import oracle

G = gbp_cases.load()
CASES = json.loads(str(G["cases"]))
INPUTS = {k[3:]: G[k].astype(np.float32) for k in G if k.startswith("in_")}


def test_fixture_cases_match_case_list():
    assert CASES == json.loads(json.dumps(gbp_cases.CASES))


def test_inputs_regenerate():
    for k, v in gbp_cases.make_inputs().items():
        np.testing.assert_array_equal(v, INPUTS[k])


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_gbp(case):
    proj = INPUTS[case["input"]]
    ref = G["out_" + case["name"]]
    got = gbp_cases.oracle_volume(oracle, proj, case["props"])
    assert got.shape == ref.shape
    store = case["props"].get("store-type", "float")
    if store in ("uchar", "ushort", "uint"):
        assert gbp_cases.integer_agrees(got, ref, proj.shape[0], int(case["props"].get("burst", 8)))
    elif store == "half" or case["props"].get("result-type") == "half":
        assert oracle.rel_l2(got, ref) < 3e-3
    else:
        assert oracle.rel_l2(got, ref) < 1e-5, oracle.rel_l2(got, ref)
