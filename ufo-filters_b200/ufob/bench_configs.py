"""Throughput of the secondary workloads (one JSON line each).

    python -m ufob.bench_configs            # general backprojection and uneven batch
    python -m ufob.bench_configs --gbp      # only the general backprojection
    python -m ufob.bench_configs --pre      # only the preprocessing stages
    python -m ufob.bench_configs --stacked  # only stacked-backproject
    python -m ufob.bench_configs --lamino   # only lamino-backproject
    python -m ufob.bench_configs --single   # only the one-slice 512^2 x 512 FBP

* general backprojection: 1024 projections of 1024^2 over 360 degrees into a
  512^3 volume, for the cone geometry (source 800 px before the axis, detector
  200 px behind it; both scale with --detector), laminography (axis tilted by 30 degrees about x,
  `axis-angle-x` = pi/6, 0 = tomography) and the parallel-beam case through the
  same task; inputs are uniform random projections (throughput does not depend
  on the values).  Each with exact FP32 interpolation weights (the default) and
  with the engine's `interpolation=texture` (the texture unit's linear filter,
  8-bit weights, as the reference samples on a GPU).
* uneven batch: 64 parallel-beam jobs with widths drawn from
  {256, 512, 1024, 1536, 2048} and 180..1800 angles (seeded), filtered and
  backprojected by one persistent launch pair captured in a CUDA graph, for
  FP32 and FP16 filtered storage.

* preprocessing (``--pre``): 1500 raw projections of 256 detector rows x 2048
  columns with one dark and one flat frame: flat-field correction (with
  absorption correction) and transpose-projections on their own (GB/s of
  algorithmic traffic: 4 B read + 4 B written per element), the filter stage
  fed by them (three passes) against the filter stage with both fused into its
  loads (one pass), and the whole parallel-beam reconstruction of the 256
  slices from the raw projections (GUPS) against the same from ready
  sinograms.

* stacked-backproject (``--stacked``): 32 slices of 2048^2 from 1500 angles
  (uniform random sinograms) in the three precision modes.

* lamino-backproject (``--lamino``): 1024 projections of 1024^2 into 512^3
  at 30 degrees from the beam (the general-backproject lamino case through the
  older task's surface).

Units are voxel-angle updates per second (GUPS); times come from CUDA events
after a warm-up call and average over repeated calls.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np


def _timeit(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def bench_gbp(reps=2, n_proj=1024, det=1024, vol=512, interpolations=("exact", "texture"),
              computes=("float", "half"), stagings=("auto",), geometries=None):
    import torch
    from . import GeneralBackprojectTask
    proj = torch.rand(n_proj, det, det, device="cuda")
    # cone distances scale with the detector (800 / 200 px at 1024 px)
    geoms = {"cone": {"source-position-y": -800.0 * det / 1024, "detector-position-y": 200.0 * det / 1024},
             "lamino_30deg": {"axis-angle-x": math.pi / 6},
             "parallel": {}}
    if geometries:
        geoms = {k: v for k, v in geoms.items() if k in geometries}
    out = []
    for (name, g), interp, ct, st in [(gi, ip, c, sg) for c in computes for ip in interpolations for sg in stagings
                                      for gi in geoms.items()]:
        t = GeneralBackprojectTask(num_projections=n_proj)
        t.set_property("interpolation", interp)
        t.set_property("compute-type", ct)
        t.set_property("staging", st)
        t.set_property("center-position-x", det / 2.0)
        t.set_property("center-position-z", det / 2.0)
        half = vol / 2.0
        t.set_property("x-region", (-half, half, 1.0))
        t.set_property("y-region", (-half, half, 1.0))
        t.set_property("region", (-half, half, 1.0))
        for k, v in g.items():
            t.set_property(k, v)
        v = t.process(proj)
        ms = _timeit(lambda: t.process(proj, out=v), reps)
        upd = float(vol) ** 3 * n_proj
        out.append({"workload": "general-backproject %s, %d projections of %d^2 -> %d^3" % (name, n_proj, det, vol),
                    "interpolation": interp, "compute_type": ct, "staging": st, "ms": round(ms, 2),
                    "gups": round(upd / ms / 1e6, 1)})
    return out


def bench_single(reps=200, seed=7, width=512, n_angles=512):
    """One 512^2 slice from 512 angles (the reference's CPU-runnable case): the whole
    fft ! filter ! ifft ! backproject call per slice, plain FP32 and FP16 pair storage."""
    import torch
    from . import F16, F32, FBP, phantom_sinogram
    from .cnn import random_ellipses
    sino = phantom_sinogram(random_ellipses(seed), width, n_angles)
    out = []
    for name, storage in (("fp32", F32), ("fp16", F16)):
        fbp = FBP(bp_props={"axis_pos": (width - 1) / 2.0}, storage=storage)
        img = fbp.process(sino)
        ms = _timeit(lambda: fbp.process(sino, out=img), reps)
        out.append({"workload": "one slice: %d px x %d angles, axis %.1f, %s storage" % (width, n_angles,
                                                                                       (width - 1) / 2.0, name),
                    "us_per_slice": round(ms * 1e3, 1), "gups": round(width * width * n_angles / ms / 1e6, 1)})
    return out


def bench_batch(reps=3, seed=2024, jobs=64):
    import torch
    from . import BF16, F16, F32, Batch
    rng = np.random.default_rng(seed)
    js, upd = [], 0
    for _ in range(jobs):
        W = int(rng.choice([256, 512, 1024, 1536, 2048]))
        P = int(rng.integers(180, 1801))
        js.append(dict(sino=torch.rand(P, W, device="cuda"), out=torch.empty(W, W, device="cuda")))
        upd += W * W * P
    out = []
    for name, storage in (("fp32", F32), ("fp16", F16), ("bf16", BF16)):
        b = Batch(storage=storage)
        ms = _timeit(lambda: b.run(js), reps)
        out.append({"workload": "uneven batch of %d jobs (seed %d), %s storage" % (jobs, seed, name),
                    "updates": upd, "ms": round(ms, 2), "gups": round(upd / ms / 1e6, 1),
                    "tile_variant": b.variant()})
    return out


def bench_pre(reps=3, n_proj=1500, rows=256, width=2048, seed=7):
    import torch
    from . import F16, FBP, QUADS, FilterTask, FlatFieldCorrectTask, TransposeProjectionsTask
    g = torch.Generator(device="cuda").manual_seed(seed)
    dark = 100 + torch.rand(rows, width, device="cuda", generator=g)
    flat = dark + 1000
    proj = dark + 900 * torch.rand(n_proj, rows, width, device="cuda", generator=g)
    ffc = FlatFieldCorrectTask(absorption_correct=1)
    f = FilterTask()
    tr = TransposeProjectionsTask(num_projections=n_proj)
    corrected = ffc.process(proj, dark, flat)
    tr.process(corrected)
    sinos = tr.sinograms
    elems = n_proj * rows * width
    out = []
    t_ffc = _timeit(lambda: ffc.process(proj, dark, flat, out=corrected), reps)
    tr2 = TransposeProjectionsTask(num_projections=n_proj)
    tr2.sinograms = sinos

    def transpose():
        tr2._next = 0
        tr2.process(corrected)
    t_tr = _timeit(transpose, reps)
    q = f.process(sinos, dtype=F16, layout=QUADS)
    t_filt = _timeit(lambda: f.process(sinos, dtype=F16, layout=QUADS, out=q), reps)
    t_fused = _timeit(lambda: f.process_projections(proj, ffc=ffc, dark=dark, flat=flat, dtype=F16, layout=QUADS,
                                                    out=q), reps)
    gb = 8.0 * elems / 1e9
    out.append({"workload": "flat-field-correct (absorption), %d projections of %dx%d" % (n_proj, rows, width),
                "ms": round(t_ffc, 3), "gbs": round(gb / t_ffc * 1e3, 1)})
    out.append({"workload": "transpose-projections, %d projections of %dx%d" % (n_proj, rows, width),
                "ms": round(t_tr, 3), "gbs": round(gb / t_tr * 1e3, 1)})
    out.append({"workload": "raw projections -> FP16 slice-quad filtered sinograms (%d x %d x %d)"
                % (rows, n_proj, width), "separate_ms": round(t_ffc + t_tr + t_filt, 3),
                "filter_only_ms": round(t_filt, 3), "fused_ms": round(t_fused, 3),
                "fused_gbs": round(gb / t_fused * 1e3, 1)})
    del q, corrected
    fbp = FBP(storage=F16)
    vol = fbp.process(sinos)
    t_sino = _timeit(lambda: fbp.process(sinos, out=vol), reps)
    t_raw = _timeit(lambda: fbp.process_projections(proj, ffc=ffc, dark=dark, flat=flat, out=vol), reps)
    upd = float(rows) * width * width * n_proj
    out.append({"workload": "parallel-beam reconstruction of %d slices %d^2 from %d projections, FP16 storage"
                % (rows, width, n_proj), "from_sinograms_gups": round(upd / t_sino / 1e6, 1),
                "from_raw_projections_gups": round(upd / t_raw / 1e6, 1)})
    return out


def bench_stacked(reps=2, Z=32, P=1500, W=2048, seed=11):
    """stacked-backproject in its three precision modes on Z slices of W^2 from P angles."""
    import torch
    from . import StackedBackprojectTask
    g = torch.Generator(device="cuda").manual_seed(seed)
    sino = torch.rand(Z, P, W, device="cuda", generator=g) - 0.5
    out = torch.empty(Z, W, W, device="cuda")
    rows = []
    for mode in ("single", "half", "int8"):
        t = StackedBackprojectTask(precision_mode=mode)
        ms = _timeit(lambda: t.process(sino, out=out), reps)
        rows.append({"workload": "stacked-backproject precision-mode=%s, %d slices %d^2 from %d angles"
                     % (mode, Z, W, P), "ms": round(ms, 2), "gups": round(float(Z) * W * W * P / ms / 1e6, 1)})
    return rows


def bench_lamino(reps=2, n_proj=1024, det=1024, vol=512):
    """lamino-backproject (30 degrees from the beam, the task's z parameter) of
    1024 projections of 1024^2 into a 512^3 volume."""
    import torch
    from . import LaminoBackprojectTask
    proj = torch.rand(n_proj, det, det, device="cuda")
    h = vol // 2
    t = LaminoBackprojectTask(num_projections=n_proj, x_region=(-h, h, 1), y_region=(-h, h, 1),
                              region=(float(-h), float(h), 1.0), center=(det / 2.0, det / 2.0),
                              lamino_angle=math.pi / 2 - math.pi / 6, overall_angle=2 * math.pi)
    v = t.process(proj)
    ms = _timeit(lambda: t.process(proj, out=v), reps)
    return [{"workload": "lamino-backproject, %d projections of %d^2 -> %d^3" % (n_proj, det, vol),
             "ms": round(ms, 2), "gups": round(float(vol) ** 3 * n_proj / ms / 1e6, 1)}]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gbp", action="store_true", help="only the general backprojection")
    ap.add_argument("--batch", action="store_true", help="only the uneven batch")
    ap.add_argument("--pre", action="store_true", help="only the preprocessing stages")
    ap.add_argument("--stacked", action="store_true", help="only stacked-backproject")
    ap.add_argument("--lamino", action="store_true", help="only lamino-backproject")
    ap.add_argument("--single", action="store_true", help="only the one-slice 512^2 x 512 FBP")
    ap.add_argument("--pre-rows", type=int, default=256, help="detector rows of the preprocessing workload")
    ap.add_argument("--projections", type=int, default=1024)
    ap.add_argument("--detector", type=int, default=1024)
    ap.add_argument("--volume", type=int, default=512)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--gbp-compute", choices=["float", "half", "both"], default="both",
                    help="compute-type(s) of the general backprojection")
    ap.add_argument("--gbp-interp", choices=["exact", "texture", "both"], default="both",
                    help="interpolation mode(s) of the general backprojection")
    ap.add_argument("--gbp-staging", choices=["auto", "texture", "both"], default="auto",
                    help="staging of the general backprojection: TMA-staged windows where the geometry "
                         "allows (auto) or texture gathers")
    ap.add_argument("--gbp-geometries", default="", help="comma-separated subset of cone,lamino_30deg,parallel")
    args = ap.parse_args(argv)
    from . import device_status
    rows = []
    only = args.gbp or args.batch or args.pre or args.stacked or args.lamino or args.single
    if args.gbp or not only:
        computes = ("float", "half") if args.gbp_compute == "both" else (args.gbp_compute,)
        interps = ("exact", "texture") if args.gbp_interp == "both" else (args.gbp_interp,)
        stagings = ("auto", "texture") if args.gbp_staging == "both" else (args.gbp_staging,)
        geoms = [g for g in args.gbp_geometries.split(",") if g] or None
        rows += bench_gbp(args.reps, args.projections, args.detector, args.volume, interps, computes, stagings, geoms)
    if args.batch or not only:
        rows += bench_batch()
    if args.pre or not only:
        rows += bench_pre(rows=args.pre_rows)
    if args.stacked or not only:
        rows += bench_stacked()
    if args.lamino or not only:
        rows += bench_lamino()
    if args.single or not only:
        rows += bench_single()
    device_status()
    for r in rows:
        print(json.dumps(r))


if __name__ == "__main__":
    main()
