"""General backprojection (parallel, cone, laminography) against the FP64 oracle.

Reference: src/ufo-general-backproject-task.c (setup :1411-1462,
get_requisition :1464-1587, process :1610-1706, generate :1708-1764,
transform chain :768-1048) and src/kernels/templates/general_bp_*.in."""
import math

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu

N, H, W = 40, 48, 64


def _proj(seed=0, n=N, h=H, w=W, smooth=False):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((n, h, w)).astype(np.float32)
    if smooth:
        yy, xx = np.mgrid[:h, :w]
        p = np.stack([np.exp(-((xx - w / 2 - 5 * math.sin(i)) ** 2 + (yy - h / 2) ** 2) / 200.0)
                      for i in range(n)]).astype(np.float32)
    return p


BASE = {"center-position-x": W / 2, "center-position-z": H / 2, "region": (-4.0, 4.0, 1.0)}

GEOMETRIES = {
    "parallel": {},
    "parallel_pi": {"overall-angle": math.pi},
    "cone": {"source-position-y": -120.0, "detector-position-y": 40.0},
    "lamino": {"axis-angle-x": math.pi / 6},
    "cone_lamino": {"source-position-y": -150.0, "detector-position-y": 20.0, "axis-angle-x": 0.3},
    "axis_roll": {"axis-angle-y": 0.05, "axis-angle-x": 0.2},
    "shifted_detector": {"detector-position-x": 3.5, "detector-position-z": -1.25},
    "shifted_cone": {"source-position-y": -120.0, "detector-position-y": 40.0, "source-position-x": 2.0,
                     "detector-position-x": -1.5},
    "detector_tilt": {"detector-angle-x": 0.1, "detector-angle-z": 0.05},
    "detector_tilt_cone": {"detector-angle-y": 0.07, "source-position-y": -120.0, "detector-position-y": 40.0},
    "volume_rotation": {"volume-angle-z": 0.3, "volume-angle-x": 0.1, "volume-angle-y": -0.05},
    "regions": {"x-region": (-20.0, 20.0, 0.5), "y-region": (-10.0, 15.0, 1.0)},
}


def run_gbp(proj, props, **opts):
    t = ufob.GeneralBackprojectTask(num_projections=proj.shape[0])
    for k, v in props.items():
        t.set_property(k, v)
    for k, v in opts.items():
        t.set_property(k, v)
    return t.process(torch.from_numpy(proj).cuda())


def oracle_gbp(proj, props, **opts):
    kw = {}
    for k, v in props.items():
        if k in ("region", "x-region", "y-region"):
            kw[k.replace("-", "_")] = tuple(v)
        elif k == "overall-angle":
            kw["overall_angle"] = v
        elif k == "parameter":
            kw["parameter"] = v
        elif k == "z":
            kw["z"] = v
        elif k == "addressing-mode":
            kw["addressing_mode"] = v
        else:
            kw[k] = v
    kw.update(opts)
    return oracle.general_backproject(proj, proj.shape[0], **kw)


@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_geometry(cuda, name):
    props = dict(BASE, **GEOMETRIES[name])
    proj = _proj(1)
    got = run_gbp(proj, props).cpu().numpy()
    ref = oracle_gbp(proj, props)
    assert got.shape == ref.shape
    tol = 1e-4 if "cone" in name else 2e-5
    assert oracle.rel_l2(got, ref) < tol, oracle.rel_l2(got, ref)


def test_per_projection_arrays(cuda):
    """Vectorised geometry: arrays with num-projections values (the reference's
    general_bp_header_vector.in path)."""
    rng = np.random.default_rng(3)
    props = dict(BASE)
    props["center-position-x"] = W / 2 + rng.uniform(-2, 2, N)
    props["detector-position-z"] = rng.uniform(-1, 1, N)
    props["axis-angle-x"] = np.full(N, 0.2)
    props["axis-angle-z"] = np.sort(rng.uniform(0, 2 * math.pi, N))
    proj = _proj(4)
    got = run_gbp(proj, props).cpu().numpy()
    assert oracle.rel_l2(got, oracle_gbp(proj, props)) < 2e-5


@pytest.mark.parametrize("param,region", [("axis-angle-x", (0.0, 0.5, 0.1)), ("center-position-x", (30.0, 34.0, 0.5)),
                                          ("detector-angle-z", (-0.02, 0.02, 0.01)),
                                          ("volume-angle-z", (0.0, 0.3, 0.1))])
def test_parameter_sweep(cuda, param, region):
    props = dict(BASE, parameter=param, region=region, z=1.5)
    proj = _proj(5)
    got = run_gbp(proj, props).cpu().numpy()
    ref = oracle_gbp(proj, props)
    assert got.shape == ref.shape
    assert oracle.rel_l2(got, ref) < 2e-5


def test_default_region_single_slice(cuda):
    proj = _proj(6)
    props = {"center-position-x": W / 2, "center-position-z": H / 2, "z": 2.0}
    got = run_gbp(proj, props).cpu().numpy()
    ref = oracle_gbp(proj, props)
    assert got.shape == (1, W, W)  # one slice of width x width by default
    assert oracle.rel_l2(got, ref) < 2e-5


def test_clamp_to_edge(cuda):
    props = dict(BASE, **GEOMETRIES["lamino"])
    proj = _proj(7)
    got = run_gbp(proj, props, **{"addressing-mode": "clamp_to_edge"}).cpu().numpy()
    ref = oracle_gbp(proj, props, addressing_mode="clamp_to_edge")
    assert oracle.rel_l2(got, ref) < 2e-5


def test_compute_double(cuda):
    props = dict(BASE, **GEOMETRIES["cone"])
    proj = _proj(8)
    got = run_gbp(proj, props, **{"compute-type": "double", "result-type": "double"}).cpu().numpy()
    assert oracle.rel_l2(got, oracle_gbp(proj, props)) < 1e-5


def test_result_half(cuda):
    props = dict(BASE, **GEOMETRIES["parallel"])
    proj = _proj(9, smooth=True)
    got = run_gbp(proj, props, **{"result-type": "half"}).cpu().numpy()
    assert oracle.rel_l2(got, oracle_gbp(proj, props)) < 3e-3


@pytest.mark.parametrize("store,tol", [("half", 3e-3), ("double", 2e-5)])
def test_store_float_types(cuda, store, tol):
    props = dict(BASE, **GEOMETRIES["cone"])
    proj = _proj(10, smooth=True)
    got = run_gbp(proj, props, **{"store-type": store}).cpu().numpy().astype(np.float64)
    ref = oracle.general_backproject_store(proj, N, store_type=store, region=(-4.0, 4.0, 1.0),
                                           **{k: v for k, v in props.items() if k != "region"})
    assert oracle.rel_l2(got, ref) < tol


@pytest.mark.parametrize("store", ["uchar", "ushort"])
def test_store_integer_gray_mapping(cuda, store):
    props = dict(BASE, **GEOMETRIES["parallel"])
    proj = _proj(11, smooth=True)
    gmin, gmax = -0.05, 0.2
    got = run_gbp(proj, props, **{"store-type": store, "gray-map-min": gmin, "gray-map-max": gmax}).cpu()
    got = got.numpy().astype(np.float64)
    ref = oracle.general_backproject_store(proj, N, store_type=store, gray_map_min=gmin, gray_map_max=gmax,
                                           region=(-4.0, 4.0, 1.0), **{k: v for k, v in props.items() if k != "region"})
    diff = np.abs(got - ref)
    # per-burst truncation can flip by one count where FP32 and FP64 straddle an integer
    assert np.mean(diff > 0) < 0.02
    assert diff.max() <= N // 8


def test_streaming_reductor(cuda):
    """process() one projection at a time, then generate() every slice; generate
    refuses output before all num-projections projections arrived (:1733-1738)."""
    props = dict(BASE, **GEOMETRIES["lamino"])
    proj = _proj(12)
    t = ufob.GeneralBackprojectTask(num_projections=N)
    for k, v in props.items():
        t.set_property(k, v)
    L = ufob.lib()
    dproj = torch.from_numpy(proj).cuda()
    ow, oh, ns = t.get_requisition(W, H)
    sl = torch.empty((oh, ow), dtype=torch.float32, device="cuda")
    for i in range(N - 1):
        ufob.check(L.ufob_gbp_process(t._h, dproj[i].data_ptr(), W, H, None))
    st = L.ufob_gbp_generate(t._h, sl.data_ptr(), 0, None)
    assert st == ufob.ERR_INVALID and b"received only" in L.ufob_last_error()
    ufob.check(L.ufob_gbp_process(t._h, dproj[N - 1].data_ptr(), W, H, None))
    ref = oracle_gbp(proj, props)
    for z in range(ns):
        ufob.check(L.ufob_gbp_generate(t._h, sl.data_ptr(), z, None))
        torch.cuda.synchronize()
        assert oracle.rel_l2(sl.cpu().numpy(), ref[z]) < 2e-5


def test_setup_errors(cuda):
    t = ufob.GeneralBackprojectTask()
    with pytest.raises(ufob.UfobError) as e:
        t.setup()
    assert e.value.status == ufob.ERR_SETUP and "Number of projections not set" in str(e.value)
    t = ufob.GeneralBackprojectTask(num_projections=10)
    t.set_property("store-type", "uchar")
    with pytest.raises(ufob.UfobError) as e:
        t.setup()
    assert "Gray mapping" in str(e.value)
    t = ufob.GeneralBackprojectTask(num_projections=10)
    t.set_property("center-position-x", [1.0, 2.0, 3.0])
    with pytest.raises(ufob.UfobError):
        t.setup()


@pytest.mark.parametrize("name", ["cone", "parallel", "lamino"])
def test_hardware_interpolation_mode(cuda, name):
    """interpolation=texture (engine property): the texture unit's linear filter with 8-bit
    weights, as the reference samples on a GPU.  Close to the exact-weight result (the weights
    differ by up to 1/512), and the default stays exact."""
    props = dict(BASE, **GEOMETRIES[name])
    proj = _proj(21, smooth=True)
    exact = run_gbp(proj, props).cpu().numpy()
    hw = run_gbp(proj, props, interpolation="texture").cpu().numpy()
    ref = oracle_gbp(proj, props)
    assert oracle.rel_l2(exact, ref) < 2e-5
    assert 1e-6 < oracle.rel_l2(hw, ref) < 1e-2
    t = ufob.GeneralBackprojectTask(num_projections=proj.shape[0])
    with pytest.raises(ufob.UfobError):
        t.set_property("interpolation", "cubic")


@pytest.mark.parametrize("name", ["cone", "parallel", "lamino", "cone_lamino", "detector_tilt"])
def test_compute_half(cuda, name):
    """compute-type half: projection samples stored as FP16 (texture gathers of 16-bit texels),
    coordinates, weights and sums in FP32.  Equal to the FP32 path on FP16-rounded projections."""
    props = dict(BASE, **GEOMETRIES[name])
    proj = _proj(31, smooth=True)
    got = run_gbp(proj, props, **{"compute-type": "half"}).cpu().numpy()
    rounded = proj.astype(np.float16).astype(np.float32)
    assert oracle.rel_l2(got, oracle_gbp(rounded, props)) < 2e-5
    assert oracle.rel_l2(got, oracle_gbp(proj, props)) < 1e-3


def test_compute_half_padded_rows_and_modes(cuda):
    """Rows whose FP16 pitch needs padding to the texture pitch alignment; clamp_to_edge
    addressing; half samples with the texture unit's linear filter; switching back to float."""
    w = 50
    props = {"center-position-x": w / 2, "center-position-z": H / 2, "region": (-3.0, 3.0, 1.0),
             "source-position-y": -120.0, "detector-position-y": 40.0}
    proj = _proj(32, w=w, smooth=False)
    rounded = proj.astype(np.float16).astype(np.float32)
    t = ufob.GeneralBackprojectTask(num_projections=proj.shape[0])
    for k, v in props.items():
        t.set_property(k, v)
    t.set_property("compute-type", "half")
    t.set_property("addressing-mode", "clamp_to_edge")
    got = t.process(torch.from_numpy(proj).cuda()).cpu().numpy()
    assert oracle.rel_l2(got, oracle_gbp(rounded, props, addressing_mode="clamp_to_edge")) < 2e-5
    t.set_property("interpolation", "texture")
    hw = t.process(torch.from_numpy(proj).cuda()).cpu().numpy()
    assert oracle.rel_l2(hw, oracle_gbp(rounded, props, addressing_mode="clamp_to_edge")) < 1e-2
    t.set_property("interpolation", "exact")
    t.set_property("compute-type", "float")
    full = t.process(torch.from_numpy(proj).cuda()).cpu().numpy()
    assert oracle.rel_l2(full, oracle_gbp(proj, props, addressing_mode="clamp_to_edge")) < 2e-5


@pytest.mark.parametrize("store,tol", [("half", 3e-3), ("float", 2e-5), ("double", 2e-5)])
def test_compute_half_with_store_types(cuda, store, tol):
    """FP16 samples combine with every floating store type: equal (within the store's precision)
    to the FP64 store semantics applied to FP16-rounded projections."""
    props = dict(BASE, **GEOMETRIES["cone"])
    proj = _proj(33, smooth=True)
    rounded = proj.astype(np.float16).astype(np.float32)
    got = run_gbp(proj, props, **{"compute-type": "half", "store-type": store}).cpu().numpy().astype(np.float64)
    ref = oracle.general_backproject_store(rounded, N, store_type=store, region=(-4.0, 4.0, 1.0),
                                           **{k: v for k, v in props.items() if k != "region"})
    assert oracle.rel_l2(got, ref) < tol


def test_compute_half_streaming_matches_one_shot(cuda):
    """Projections passed one by one (process, then generate per slice) with FP16 samples give
    the one-shot volume."""
    props = dict(BASE, **GEOMETRIES["lamino"])
    proj = _proj(34, smooth=True)
    one = run_gbp(proj, props, **{"compute-type": "half"}).cpu().numpy()
    t = ufob.GeneralBackprojectTask(num_projections=N)
    for k, v in props.items():
        t.set_property(k, v)
    t.set_property("compute-type", "half")
    L = ufob.lib()
    dproj = torch.from_numpy(proj).cuda()
    ow, oh, ns = t.get_requisition(W, H)
    for i in range(N):
        ufob.check(L.ufob_gbp_process(t._h, dproj[i].data_ptr(), W, H, None))
    sl = torch.empty((oh, ow), dtype=torch.float32, device="cuda")
    for z in range(ns):
        ufob.check(L.ufob_gbp_generate(t._h, sl.data_ptr(), z, None))
        torch.cuda.synchronize()
        assert oracle.rel_l2(sl.cpu().numpy(), one[z]) < 1e-6


@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_staged_windows_match_texture_path(cuda, name):
    """The TMA-staged kernel (detector windows in shared memory, for geometries whose u does not
    depend on z) and the texture-gather kernel use the same footprint rule and exact FP32
    weights; the staged kernel forms v as one affine function of z per column, so the two
    differ by FP32 coordinate rounding only.  Both agree with the oracle on every geometry (the
    staged path declines the tilted ones and runs the texture path itself)."""
    props = dict(BASE, **GEOMETRIES[name])
    props["region"] = (-12.0, 12.0, 1.0)  # several z tiles of 8 voxels, the last one partial
    proj = _proj(11)
    staged = run_gbp(proj, props).cpu().numpy()
    tex = run_gbp(proj, props, staging="texture").cpu().numpy()
    ref = oracle_gbp(proj, props)
    tol = 1e-4 if "cone" in name else 2e-5
    assert oracle.rel_l2(staged, ref) < tol
    assert oracle.rel_l2(staged, tex) < 1e-5


def test_staged_windows_large_cone(cuda):
    """Cone beam of 360 projections of 256^2 into 128 x 96 x 40 voxels, an odd region that leaves
    partial tiles in x, y and z, against the oracle and the texture-gather kernel."""
    n, det = 360, 256
    rng = np.random.default_rng(12)
    proj = rng.uniform(0.0, 1.0, (n, det, det)).astype(np.float32)
    props = {"center-position-x": det / 2.0 + 0.3, "center-position-z": det / 2.0 - 0.7,
             "source-position-y": -300.0, "detector-position-y": 60.0,
             "x-region": (-64.0, 64.0, 1.0), "y-region": (-40.0, 56.0, 1.0), "region": (-20.0, 20.0, 1.0)}
    staged = run_gbp(proj, props).cpu().numpy()
    tex = run_gbp(proj, props, staging="texture").cpu().numpy()
    assert staged.shape == (40, 96, 128)
    ref = oracle_gbp(proj, props)
    assert oracle.rel_l2(staged, ref) < 1e-4
    assert oracle.rel_l2(staged, tex) < 1e-5
