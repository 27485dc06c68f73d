"""Generate the golden fixtures in this folder from the reference itself.

The reference's `filter`, `backproject`, `general-backproject`, `lamino-backproject` and
`stacked-backproject` task sources and its OpenCL kernels (with the flat-field and cone-beam weight kernels) are compiled for
the CPU by oracle/ref.mk (oracle/_ref/libufo_ref.so, see oracle/reference.py); the kernels
general-backproject generates at run time, and the lamino kernels its build generates, are compiled
when the tasks ask for them.  This script runs them on seeded inputs and
stores inputs and outputs.  Run it where the reference sources are present:

    make -C oracle -f ref.mk && python tests/golden/make_golden.py [fbp|pre|gbp|lamino|stacked ...]
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, ".."))
import gbp_cases  # noqa: E402
import lamino_cases  # noqa: E402
import stacked_cases  # noqa: E402
import oracle  # noqa: E402  (phantom generators only)
import reference  # noqa: E402

FILTER_CASES = [
    dict(filter="ramp-fromreal"), dict(filter="ramp"), dict(filter="butterworth", cutoff=0.3, order=6.0),
    dict(filter="faris-byer", tau=0.2, theta=0.7), dict(filter="hamming", cutoff=0.4), dict(filter="bh3"),
    dict(filter="ramp-fromreal", scale=1.7), dict(filter="butterworth", scale=0.5),
]
CHAIN_CASES = [dict(), dict(size_x=128, crop_width=100), dict(size_x=128), dict(filter="hamming", cutoff=0.4),
               dict(filter="ramp")]
BP_CASES = [dict(), dict(axis_pos=31.5), dict(axis_pos=30.25, angle_step=0.05, angle_offset=0.3),
            dict(roi_x=10, roi_y=5, roi_width=40, roi_height=30), dict(num_projections=80, offset=20),
            dict(mode="nearest", roi_x=3, roi_width=50, roi_height=50)]


def main():
    out = {}
    for i, c in enumerate(FILTER_CASES):
        for n in (8, 64, 256):
            out["coeff_%d_%d" % (i, n)] = reference.filter_coefficients(n, **c)
    rng = np.random.default_rng(1234)
    sino = rng.standard_normal((17, 64)).astype(np.float32)
    out["chain_input"] = sino
    for i, c in enumerate(CHAIN_CASES):
        out["chain_%d" % i] = reference.fft_filter_ifft(sino, **c)
    bp_in = rng.standard_normal((45, 64)).astype(np.float32)
    out["bp_input"] = bp_in
    for i, c in enumerate(BP_CASES):
        out["bp_%d" % i] = reference.backproject(bp_in, **c)
    # FBP of an analytic ellipse phantom, 128 px, 128 angles (the C0 recipe at a quarter size)
    ell = oracle.random_ellipses(7)
    W = P = 128
    fsino = oracle.ellipse_sinogram(ell, W, np.arange(P) * math.pi / P).astype(np.float32)
    out["fbp_input"] = fsino
    out["fbp_output"] = reference.fbp(fsino, axis_pos=63.5)
    img = oracle.ellipse_image(ell, 64).astype(np.float32)
    out["fp_input"] = img
    out["fp_output"] = reference.forwardproject(img, 30, 32.0, math.pi / 30)
    path = os.path.join(HERE, "reference_fbp.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


FFC_CASES = [dict(), dict(absorption_correct=True), dict(absorption_correct=True, fix_nan_and_inf=True),
             dict(dark_scale=0.5, flat_scale=1.5)]
CONE_CASES = [dict(center_position_x=20.5, center_position_z=9.0, source_distance=300.0, detector_distance=100.0),
              dict(center_position_x=17.25, center_position_z=11.5, source_distance=150.0, detector_distance=60.0,
                   axis_angle_x=0.4)]


def pre_golden():
    """flat-field-correct and cone-beam-projection-weight kernels of the reference (ffc.cl,
    conebeam.cl) on seeded frames; the cone arguments are the task's FP32 host arithmetic."""
    rng = np.random.default_rng(77)
    H, W = 12, 40
    dark = rng.uniform(90, 110, (H, W)).astype(np.float32)
    flat = (dark + rng.uniform(800, 1200, (H, W))).astype(np.float32)
    data = (dark + rng.uniform(50, 1000, (3, H, W))).astype(np.float32)
    data[0, 0, :3] = dark[0, :3]  # zero transmission
    out = {"ffc_dark": dark, "ffc_flat": flat, "ffc_data": data}
    for i, c in enumerate(FFC_CASES):
        out["ffc_%d" % i] = reference.flat_field_correct(data, dark, flat, **c)
    proj = rng.standard_normal((H, W)).astype(np.float32)
    out["cone_input"] = proj
    for i, c in enumerate(CONE_CASES):
        cx, cz, sd, od, mr, cs = oracle.cone_weight_params(0, **c)
        out["cone_%d" % i] = reference.weight_projection(proj, cx, cz, sd, od, mr, cs)
    path = os.path.join(HERE, "reference_pre.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def gbp_golden():
    """The reference's general-backproject task on the cases of tests/gbp_cases.py."""
    inputs = gbp_cases.make_inputs()
    out = {"in_" + k: (v.astype(np.float16) if k == "d" else v) for k, v in inputs.items()}
    out["cases"] = np.array(json.dumps(gbp_cases.CASES))
    for c in gbp_cases.CASES:
        vol = reference.general_backproject(inputs[c["input"]], c["props"],
                                            max_alloc_slices=c.get("max_alloc_slices", 0))
        out["out_" + c["name"]] = vol
        print("  %-28s %s %s" % (c["name"], vol.shape, vol.dtype))
    path = os.path.join(HERE, "reference_gbp.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def lamino_golden():
    """The reference's lamino-backproject task on the cases of tests/lamino_cases.py."""
    proj = lamino_cases.make_input()
    out = {"input": proj, "cases": np.array(json.dumps(lamino_cases.CASES))}
    for c in lamino_cases.CASES:
        vol = reference.lamino_backproject(proj, c["props"])
        out["out_" + c["name"]] = vol
        print("  %-16s %s" % (c["name"], vol.shape))
    path = os.path.join(HERE, "reference_lamino.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def stacked_golden():
    """The reference's stacked-backproject task on the cases of tests/stacked_cases.py."""
    sino = stacked_cases.make_input(oracle)
    out = {"input": sino, "cases": np.array(json.dumps(stacked_cases.CASES))}
    for c in stacked_cases.CASES:
        out["out_" + c["name"]] = reference.stacked_backproject(sino, c["props"])
        print("  %-10s %s" % (c["name"], out["out_" + c["name"]].shape))
    path = os.path.join(HERE, "reference_stacked.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    which = sys.argv[1:] or ["fbp", "pre", "gbp", "lamino", "stacked"]
    if "fbp" in which:
        main()
    if "pre" in which:
        pre_golden()
    if "gbp" in which:
        gbp_golden()
    if "lamino" in which:
        lamino_golden()
    if "stacked" in which:
        stacked_golden()
