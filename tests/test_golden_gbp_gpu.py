"""The CUDA general backprojector against the reference's own general-backproject task.

tests/golden/reference_gbp.npz holds the volumes the reference task computes with the kernel its
make_kernel generates (src/ufo-general-backproject-task.c:1069-1180, compiled for the CPU by
oracle/refshim; tests/golden/make_golden.py) on the cases of tests/gbp_cases.py: parallel, cone,
laminography, tilted axis, shifted/tilted detectors, rotated volumes, regions, per-projection
geometry, parameter sweeps, compute/result/store types, bursts, chunked volumes, odd sizes and
configuration 2 (cone 800/200 px, laminography 30 degrees) at reduced size.  The engine runs each
case through the task surface (ufob.GeneralBackprojectTask -> ufob_gbp_* C ABI)."""
import json

import numpy as np
import pytest
import torch

import gbp_cases
import oracle
import ufob

pytestmark = pytest.mark.gpu
G = gbp_cases.load()
CASES = json.loads(str(G["cases"]))
INPUTS = {k[3:]: G[k].astype(np.float32) for k in G if k.startswith("in_")}


def run_engine(proj, props):
    t = ufob.GeneralBackprojectTask(num_projections=proj.shape[0])
    for k, v in props.items():
        t.set_property(k, v)
    return t.process(torch.from_numpy(proj).cuda()).cpu().numpy()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_engine_matches_reference_gbp(cuda, case):
    proj = INPUTS[case["input"]]
    ref = G["out_" + case["name"]]
    got = run_engine(proj, case["props"])
    assert got.shape == ref.shape and got.dtype == ref.dtype
    store = case["props"].get("store-type", "float")
    if store in ("uchar", "ushort", "uint"):
        assert gbp_cases.integer_agrees(got, ref, proj.shape[0], int(case["props"].get("burst", 8)))
    else:
        err = oracle.rel_l2(got.astype(np.float64), ref.astype(np.float64))
        assert err < gbp_cases.tolerance(case), err


@pytest.mark.parametrize("name", ["c2_cone", "c2_lamino", "c2_parallel"])
def test_engine_half_samples_near_reference(cuda, name):
    """compute-type half (FP16 projection samples, FP32 arithmetic) stays within 1e-3 of the
    reference's FP32 volume on the configuration-2 geometries."""
    case = [c for c in CASES if c["name"] == name][0]
    props = dict(case["props"], **{"compute-type": "half"})
    got = run_engine(INPUTS[case["input"]], props)
    assert oracle.rel_l2(got, G["out_" + name]) < 1e-3
