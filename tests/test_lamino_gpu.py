"""lamino-backproject on the GPU against the oracle.

Reference: src/ufo-lamino-backproject-task.c:164-517 and the kernels generated
from src/kernels/templates/{z,center,lamino,roll}_template.in.  The engine runs
the task on the general backprojector's kernel (one affine table per slice and
projection, FP32 texture gathers with exact weights); tolerance 2e-5 relative
L2 against the FP64 oracle built from the same FP32 scalars."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob
from test_oracle_lamino import tomographic_limit_case

pytestmark = pytest.mark.gpu

N, H, W = 48, 40, 64
BASE = dict(num_projections=N, x_region=(-24, 24, 1), y_region=(-20, 28, 2), center=(W / 2 + 0.25, H / 2 - 1.5),
            projection_offset=(1, -2), lamino_angle=0.6)

CASES = {
    "z": dict(region=(-6.0, 6.0, 1.5)),
    "z_roll": dict(region=(-4.0, 4.0, 1.0), roll_angle=0.12),
    "x_center": dict(region=(30.0, 36.0, 1.0), parameter="x-center", z=2.0),
    "lamino_sweep": dict(region=(0.3, 0.9, 0.1), parameter="lamino-angle", z=-3.0),
    "roll_sweep": dict(region=(-0.2, 0.2, 0.1), parameter="roll-angle", z=1.0),
    "tomo_fixed": dict(region=(-2.0, 2.0, 1.0), tomo_angle=0.4),
    "edge": dict(region=(-2.0, 2.0, 1.0), addressing_mode="clamp_to_edge"),
    "overall": dict(region=(-2.0, 2.0, 1.0), overall_angle=2 * math.pi),
}


def _proj(seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((N, H, W)).astype(np.float32)
    k = np.ones(5, np.float32) / 5  # smooth so that the linear interpolation is well conditioned
    p = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 2, p)
    return np.ascontiguousarray(np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 1, p).astype(np.float32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_lamino_matches_oracle(cuda, name):
    props = dict(BASE, **CASES[name])
    proj = _proj(hash(name) % 1000)
    t = ufob.LaminoBackprojectTask(**props)
    got = t.process(torch.from_numpy(proj).cuda()).cpu().numpy()
    ref = oracle.lamino_backproject(proj, **props)
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < 2e-5, oracle.rel_l2(got, ref)


def test_lamino_streaming_equals_run(cuda):
    props = dict(BASE, **CASES["z_roll"])
    proj = torch.from_numpy(_proj(3)).cuda()
    a = ufob.LaminoBackprojectTask(**props).process(proj)
    t = ufob.LaminoBackprojectTask(**props)
    for i in range(N - 1):
        t.push(proj[i])
    with pytest.raises(ufob.UfobError):  # not all projections yet
        t.generate()
    t.push(proj[N - 1])
    b = t.generate()
    assert torch.equal(a, b)
    with pytest.raises(ufob.UfobError):  # generate() gives the volume once
        t.generate()


def test_lamino_tomographic_limit_is_backproject(cuda):
    sinos, proj, props = tomographic_limit_case()
    vol = ufob.LaminoBackprojectTask(**props).process(torch.from_numpy(proj).cuda())
    ref = ufob.BackprojectTask(axis_pos=sinos.shape[-1] / 2 + 0.5).process(torch.from_numpy(sinos).cuda())
    assert oracle.rel_l2(vol.cpu().numpy(), ref.cpu().numpy()) < 1e-5
