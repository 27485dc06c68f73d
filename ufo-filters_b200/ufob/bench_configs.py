"""Throughput of the secondary workloads (one JSON line each).

    python -m ufob.bench_configs            # general backprojection and uneven batch
    python -m ufob.bench_configs --gbp      # only the general backprojection

* general backprojection: 1024 projections of 1024^2 over 360 degrees into a
  512^3 volume, for the cone geometry (source 800 px before the axis, detector
  200 px behind it), laminography (axis tilted by 30 degrees about x,
  `axis-angle-x` = pi/6, 0 = tomography) and the parallel-beam case through the
  same task; inputs are uniform random projections (throughput does not depend
  on the values).
* uneven batch: 64 parallel-beam jobs with widths drawn from
  {256, 512, 1024, 1536, 2048} and 180..1800 angles (seeded), filtered and
  backprojected by one persistent launch pair captured in a CUDA graph, for
  FP32 and FP16 filtered storage.

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


def bench_gbp(reps=2, n_proj=1024, det=1024, vol=512):
    import torch
    from . import GeneralBackprojectTask
    proj = torch.rand(n_proj, det, det, device="cuda")
    geoms = {"cone": {"source-position-y": -800.0, "detector-position-y": 200.0},
             "lamino_30deg": {"axis-angle-x": math.pi / 6},
             "parallel": {}}
    out = []
    for name, g in geoms.items():
        t = GeneralBackprojectTask(num_projections=n_proj)
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
                    "ms": round(ms, 2), "gups": round(upd / ms / 1e6, 1)})
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


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gbp", action="store_true", help="only the general backprojection")
    ap.add_argument("--batch", action="store_true", help="only the uneven batch")
    ap.add_argument("--projections", type=int, default=1024)
    ap.add_argument("--detector", type=int, default=1024)
    ap.add_argument("--volume", type=int, default=512)
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args(argv)
    from . import device_status
    rows = []
    if not args.batch:
        rows += bench_gbp(args.reps, args.projections, args.detector, args.volume)
    if not args.gbp:
        rows += bench_batch()
    device_status()
    for r in rows:
        print(json.dumps(r))


if __name__ == "__main__":
    main()
