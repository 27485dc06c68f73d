"""Cases of the general-backproject golden fixtures (tests/golden/reference_gbp.npz).

Each case is a set of the reference task's properties (src/ufo-general-backproject-task.c:2087-2359)
applied to one of four seeded projection stacks.  tests/golden/make_golden.py runs the reference's
own task over them (its generated kernel compiled for the CPU, oracle/reference.py) and stores the
volumes; the oracle (CPU) and the CUDA engine (GPU) are checked against those volumes."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_gbp.npz")


def make_inputs():
    """Projection stacks [n, height, width]: a (noise, 24 x 32 x 48), b (smooth, same shape),
    c (noise at odd sizes, 17 x 21 x 37), d (smooth, 96 x 64 x 64: configuration 2 at 1/16 of the
    detector and 1/8 of the volume side)."""
    rng = np.random.default_rng(2024)
    a = rng.standard_normal((24, 32, 48)).astype(np.float32)
    yy, xx = np.mgrid[:32, :48]
    b = np.stack([np.exp(-((xx - 24 - 5 * math.sin(i)) ** 2 + (yy - 16) ** 2) / 150.0)
                  for i in range(24)]).astype(np.float32)
    c = rng.standard_normal((17, 21, 37)).astype(np.float32)
    yy, xx = np.mgrid[:64, :64]
    blobs = rng.uniform([-12, -12, 4, 0.3], [12, 12, 8, 1.0], (6, 4))  # x, z, sigma, amplitude
    d = []
    for i in range(96):
        th = 2 * math.pi * i / 96
        img = np.zeros((64, 64))
        for bx, bz, s, amp in blobs:
            u = 32 + bx * math.cos(th) - (bx * 0.5) * math.sin(th)
            img += amp * np.exp(-((xx - u) ** 2 + (yy - 32 - bz) ** 2) / (2 * s * s))
        d.append(img)
    d = np.stack(d).astype(np.float16).astype(np.float32)  # exact in FP16 (stored that way)
    return {"a": a, "b": b, "c": c, "d": d}


BASE = {"center-position-x": 24.0, "center-position-z": 16.0, "region": [-3.0, 3.0, 1.0]}
CONE = {"source-position-y": -120.0, "detector-position-y": 40.0}
D_BASE = {"center-position-x": 32.0, "center-position-z": 32.0, "x-region": [-16.0, 16.0, 1.0],
          "y-region": [-16.0, 16.0, 1.0], "region": [-16.0, 16.0, 1.0]}


def _cases():
    rng = np.random.default_rng(7)
    geoms = {
        "parallel": {},
        "parallel_pi": {"overall-angle": math.pi},
        "negative_overall": {"overall-angle": -math.pi},
        "cone": dict(CONE),
        "lamino": {"axis-angle-x": math.pi / 6},
        "cone_lamino": {"source-position-y": -150.0, "detector-position-y": 20.0, "axis-angle-x": 0.3},
        "axis_roll": {"axis-angle-y": 0.05, "axis-angle-x": 0.2},
        "shifted_detector": {"detector-position-x": 3.5, "detector-position-z": -1.25},
        "shifted_cone": dict(CONE, **{"source-position-x": 2.0, "detector-position-x": -1.5}),
        "detector_tilt": {"detector-angle-x": 0.1, "detector-angle-z": 0.05},
        "detector_tilt_cone": dict(CONE, **{"detector-angle-y": 0.07}),
        "volume_rotation": {"volume-angle-z": 0.3, "volume-angle-x": 0.1, "volume-angle-y": -0.05},
        "regions": {"x-region": [-20.0, 20.0, 0.5], "y-region": [-10.0, 15.0, 1.0]},
        "clamp_to_edge": {"axis-angle-x": math.pi / 6, "addressing-mode": "clamp_to_edge"},
    }
    cases = [dict(name=k, input="a", props=dict(BASE, **v)) for k, v in geoms.items()]
    n = 24
    cases.append(dict(name="vector_parallel", input="a", props=dict(
        BASE, **{"center-position-x": list(24 + rng.uniform(-2, 2, n)),
                 "detector-position-z": list(rng.uniform(-1, 1, n)), "axis-angle-x": [0.2] * n,
                 "axis-angle-z": list(np.sort(rng.uniform(0, 2 * math.pi, n)))})))
    cases.append(dict(name="vector_cone", input="a", props=dict(
        BASE, **{"source-position-y": list(rng.uniform(-130, -110, n)), "detector-position-y": 40.0,
                 "center-position-x": list(24 + rng.uniform(-1, 1, n))})))
    cases.append(dict(name="vector_detector_tilt", input="a", props=dict(
        BASE, **{"detector-angle-x": list(rng.uniform(-0.1, 0.1, n)), "volume-angle-z": list(rng.uniform(0, 0.2, n))})))
    sweeps = [("axis-angle-x", [0.0, 0.5, 0.1], {}), ("center-position-x", [22.0, 26.0, 0.5], {}),
              ("detector-angle-z", [-0.02, 0.02, 0.01], {}), ("volume-angle-z", [0.0, 0.3, 0.1], {}),
              ("detector-position-y", [30.0, 50.0, 5.0], CONE), ("source-position-x", [-2.0, 2.0, 1.0], CONE),
              ("detector-position-x", [-2.0, 2.0, 1.0], {})]
    for param, region, extra in sweeps:
        cases.append(dict(name="sweep_" + param, input="a",
                          props=dict(BASE, **extra, parameter=param, region=region, z=1.5)))
    cases.append(dict(name="default_region", input="a",
                      props={"center-position-x": 24.0, "center-position-z": 16.0, "z": 2.0}))
    cases.append(dict(name="compute_double", input="a",
                      props=dict(BASE, **CONE, **{"compute-type": "double", "result-type": "double"})))
    cases.append(dict(name="result_half", input="b", props=dict(BASE, **{"result-type": "half"})))
    cases.append(dict(name="store_half", input="b", props=dict(BASE, **CONE, **{"store-type": "half"})))
    cases.append(dict(name="store_double", input="b", props=dict(BASE, **CONE, **{"store-type": "double"})))
    for st in ("uchar", "ushort"):
        cases.append(dict(name="store_" + st, input="b", props=dict(
            BASE, **{"store-type": st, "gray-map-min": -0.05, "gray-map-max": 0.2})))
    cases.append(dict(name="burst_5", input="a", props=dict(BASE, **CONE, burst=5)))
    cases.append(dict(name="burst_16_lamino", input="a", props=dict(BASE, burst=16, **{"axis-angle-x": 0.4})))
    cases.append(dict(name="chunked_cone", input="a", props=dict(BASE, **CONE), max_alloc_slices=2))
    cases.append(dict(name="odd_sizes", input="c", props={"center-position-x": 18.3, "center-position-z": 10.0,
                                                          "region": [-1.0, 2.0, 1.0]}))
    cases.append(dict(name="c2_cone", input="d", props=dict(
        D_BASE, **{"source-position-y": -100.0, "detector-position-y": 25.0})))
    cases.append(dict(name="c2_lamino", input="d", props=dict(D_BASE, **{"axis-angle-x": math.pi / 6})))
    cases.append(dict(name="c2_parallel", input="d", props=dict(D_BASE)))
    return cases


CASES = _cases()
FLOAT_TOL = 1e-4  # the engine's exact-weight FP32 path against the reference's own kernel


def is_cone(props):
    return any("source-position-y" == k for k in props)


def tolerance(case):
    """Relative-L2 bound of the CUDA engine against the reference's volume: the FP32 paths within
    1e-4 (cone) / 2e-5; half results or stores within FP16 rounding."""
    p = case["props"]
    if p.get("result-type") == "half" or p.get("store-type") == "half":
        return 3e-3
    return FLOAT_TOL if is_cone(p) else 2e-5


def integer_agrees(got, ref, n_proj, burst=8):
    """Integer store types add a truncated, gray-mapped burst sum per burst of projections, so a
    voxel whose burst sum straddles an integer in FP32 on one side and the other elsewhere differs
    by one count per burst: few voxels may differ, and by at most one count per burst."""
    diff = np.abs(np.asarray(got, np.float64) - np.asarray(ref, np.float64))
    return np.mean(diff > 0) < 0.02 and diff.max() <= max(1, n_proj // burst)


def oracle_kwargs(props):
    """The oracle's keyword form of a property set (oracle.general_backproject[_store])."""
    kw = {}
    for k, v in props.items():
        if k in ("region", "x-region", "y-region"):
            kw[k.replace("-", "_")] = tuple(v)
        elif k in ("overall-angle", "addressing-mode", "store-type", "gray-map-min", "gray-map-max"):
            kw[k.replace("-", "_")] = v
        elif k in ("compute-type", "result-type"):
            continue
        else:
            kw[k] = v
    return kw


def oracle_volume(oracle, proj, props):
    kw = oracle_kwargs(props)
    store = kw.pop("store_type", None)
    burst = int(kw.pop("burst", 8))
    if store and store != "float":
        return oracle.general_backproject_store(proj, proj.shape[0], store_type=store, burst=burst, **kw)
    kw.pop("gray_map_min", None)
    kw.pop("gray_map_max", None)
    return oracle.general_backproject(proj, proj.shape[0], **kw)


def load():
    return dict(np.load(GOLDEN))
