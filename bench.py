#!/usr/bin/env python
"""Benchmark of the B200 FBP engine on the batched parallel-beam workload:
a stack of 2048 sinograms, each 2048 detector bins x 1500 angles on [0, pi),
filtered (fft ! filter ! ifft, ramp-fromreal) and backprojected to 2048 x 2048
slices.  Metric: voxel-angle updates per second (GUPS), for plain FP32 and for
FP16 filtered-sinogram storage with FP32 accumulation (slice-quad cells), each with
its relative L2 error against the FP64 oracle on a seeded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ufob|reference]

One step = one pass of the engine over the whole stack (inputs resident in
HBM).  Multi-GPU: one process per GPU (torchrun); every rank reconstructs its
own full stack (independent slices, no collective in the data path: weak
scaling); the step time is the max over ranks.  Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ufo-filters_b200"))

METRIC = "FBP GUPS (voxel·angle updates/s), 2048²×1500, 1 B200; chosen vs plain at error"
HBM_FALLBACK_GBS = 6650.0  # copy bandwidth measured earlier on this pool's B200s, used without MEASURED_PEAKS.json
WORKLOAD = "batched parallel-beam FBP: 2048 slices x 2048 px x 1500 angles on [0, pi), float32"
I0 = 1.0e4  # photons per ray (Beer-Lambert + Poisson noise)


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ufob", "reference"], default="ufob")
    ap.add_argument("--slices", type=int, default=2048)
    ap.add_argument("--width", type=int, default=2048)
    ap.add_argument("--angles", type=int, default=1500)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-slices", type=int, default=0, help="0 = as many as host memory allows (<= --slices)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other four workloads' table")
    return ap.parse_args()


# ----------------------------------------------------------------------------- synthetic input

def random_ellipsoids(seed, n=50, semi=(0.05, 0.4), density=(-0.5, 1.0)):
    """50 random ellipsoids: centres uniform in the unit ball, semi-axes U[0.05, 0.4],
    rotation about z U[0, pi), densities U[-0.5, 1]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v *= rng.uniform(0, 1, (n, 1)) ** (1.0 / 3.0)
    ell = np.concatenate([v, rng.uniform(*semi, (n, 3)), rng.uniform(0, math.pi, (n, 1)),
                          rng.uniform(*density, (n, 1))], axis=1)
    return np.ascontiguousarray(ell, dtype=np.float64)


def make_stack(ufob, torch, nz, P, W, seed, device, chunk=64):
    """Noisy sinogram stack [nz, P, W] on the device: analytic ellipsoid line
    integrals (unit-ball phantom, radius W/2 px), Beer-Lambert with I0 photons,
    Poisson noise, -log, back to pixel-length units."""
    ell = random_ellipsoids(seed)
    scale = W / 2.0
    stack = torch.empty((nz, P, W), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    for z0 in range(0, nz, chunk):
        n = min(chunk, nz - z0)
        e = ell.copy()
        e[:, 2] -= (z0 + 0.5 * n - 0.5 * nz) / scale  # slice heights of this chunk within the stack
        ufob.phantom_stack(e, W, P, n, out=stack[z0:z0 + n])
        s = stack[z0:z0 + n]
        counts = torch.poisson(I0 * torch.exp(-s / scale), generator=gen)
        s.copy_(-torch.log(torch.clamp(counts, min=0.5) / I0) * scale)
    torch.cuda.synchronize()
    return stack


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, power, reasons = [], None, [], set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"],
                                 f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "power_w_median": statistics.median(power) if power else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------- CPU leg (oracle)

def cpu_leg(stack_host_slices, slice_ids, roi, P, W, gpu_rois):
    """CPU baseline and error references.  The oracle (C restatement of the
    reference's fft ! filter ! ifft ! backproject, OpenMP on all host cores)
    reconstructs a fixed ROI of the sampled slices in FP64: the reference for
    the error report.  The reference's own filter/backproject code compiled for
    the CPU reconstructs the same ROI: its wall time gives the CPU GUPS and its
    output the second error reference (the plain form must match it within
    1e-4 relative L2)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    import reference
    rx, ry, rw, rh = roi
    refs = []
    for s in stack_host_slices:  # FP64 oracle: the error reference
        filt = oracle.fft_filter_ifft(s).astype(np.float32)
        refs.append(oracle.backproject(filt, roi_x=rx, roi_y=ry, roi_width=rw, roi_height=rh))
    # timed: the reference's own filter/backproject code on the host cores where its CPU build
    # is present, else the oracle, on the whole slices (about 10 s of CPU work: 4 x 2048^2 x 1500
    # updates at ~2 GUPS); the error ROI is cut from them
    impl = reference if reference.available() else oracle
    tw = W
    tx, ty = min(max(rx - (tw - rw) // 2, 0), W - tw), min(max(ry - (tw - rh) // 2, 0), W - tw)
    outs = []
    t0 = time.perf_counter()
    for s in stack_host_slices:
        filt = impl.fft_filter_ifft(s).astype(np.float32)
        big = impl.backproject(filt, roi_x=tx, roi_y=ty, roi_width=tw, roi_height=tw)
        outs.append(big[ry - ty:ry - ty + rh, rx - tx:rx - tx + rw])
    dt = time.perf_counter() - t0
    updates = len(stack_host_slices) * tw * tw * P

    def rel(a, b):
        return float(np.linalg.norm(np.stack(a) - np.stack(b)) / np.linalg.norm(np.stack(b)))
    errors = {k: {"rel_l2_vs_fp64": rel(v, refs)} for k, v in gpu_rois.items()}
    if impl is reference:
        for k, v in gpu_rois.items():
            errors[k]["rel_l2_vs_reference"] = rel(v, outs)
    cores = os.cpu_count()
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    kind = "reference" if impl is reference else "port"
    what = ("reference filter/backproject tasks and kernels compiled for the CPU (OpenMP)" if kind == "reference"
            else "FP64 oracle")
    return {"value": updates / dt / 1e9, "unit": "GUPS", "cores": cores, "kind": kind,
            "sample": "%s: fft/filter/ifft of %d full slices + backprojection of a %dx%d ROI (%d angles), "
                      "%.2e updates, %.1f s" % (what, len(stack_host_slices), tw, tw, P, updates, dt)}, errors


def reference_arm(args):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores, on a bounded sample of the same workload per step."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import reference
    if int(os.environ.get("RANK", "0")) != 0:
        return
    W, P = args.width, args.angles
    ell = random_ellipsoids(args.seed)
    ell2 = oracle.ellipsoid_slice_ellipses(ell, args.slices // 2, args.slices, W / 2.0)
    sino = oracle.ellipse_sinogram(ell2, W, np.arange(P) * math.pi / P).astype(np.float32)
    # one step = fft ! filter ! ifft and backprojection of one whole slice (the filter's cost is
    # spread over the slice's updates as in the workload; ~3 s on 16 cores)
    side = W
    roi = (0, 0, side, side)
    impl = reference if reference.available() else oracle
    kind = "reference" if impl is reference else "port"
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        filt = impl.fft_filter_ifft(sino).astype(np.float32)
        impl.backproject(filt, roi_x=roi[0], roi_y=roi[1], roi_width=side, roi_height=side)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    dt = statistics.mean(times)
    upd = side * side * P
    val = upd / dt / 1e9
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "GUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if kind == "reference" else "f64",
            "data": "synthetic: slice of the 50-ellipsoid phantom, analytic line integrals",
            "config": {"workload": WORKLOAD, "sample_per_step": "one slice of %d bins x %d angles filtered and "
                       "backprojected to %dx%d" % (W, P, side, side)},
            "cpu_baseline": {"value": val, "unit": "GUPS", "cores": cores, "kind": kind,
                             "sample": "one %d x %d slice from %d angles per step (%.2e updates)" % (side, side, P, upd)},
            "e2e": {"value": val, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": ("the reference's filter and backproject task sources and OpenCL kernels compiled for the "
                     "host CPU through GLib/OpenCL/ufo-core shims (OpenMP over work-items, FP64 FFT in place of "
                     "oclfft); ufo-core and an OpenCL CPU runtime are absent on this box"
                     if kind == "reference" else
                     "FP64 CPU restatement of the reference path (the reference's CPU build is absent)")}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- main arm

def read_profile_traffic(name):
    """Per-update DRAM bytes of a kernel from its committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_update:\s*([0-9.eE+-]+)", text)
    return float(m.group(1)) if m else None


def _event_ms(torch, fn, reps):
    """Mean CUDA-event time (ms) of reps calls after one warm-up call, on torch's current
    stream (the stream the engine's Python objects launch on)."""
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


C2_GEOMETRIES = {"cone": {"source-position-y": -800.0, "detector-position-y": 200.0},
                 "lamino_30deg": {"axis-angle-x": math.pi / 6},
                 "parallel": {}}


def run_configs(ufob, torch, dev, seed):
    """The other four workloads on this GPU, timed with CUDA events: one 512^2
    slice (512 angles), general backprojection of 1024 projections of 1024^2
    into 512^3 (cone, laminography 30 degrees, parallel), the 64-job uneven
    batch, and the learned 90-angle path against dense FBP.  Returns the table
    and the host copies of sampled outputs that the CPU leg checks."""
    import numpy as np
    from ufob.cnn import PairMaker, SparseViewNet, random_ellipses, rel_l2
    from ufob.train_cnn import time_paths
    table, checks = {}, {}

    # configuration 0: one 512^2 slice from 512 angles, axis 255.5 (10 random ellipses)
    W0 = P0 = 512
    sino0 = ufob.phantom_sinogram(random_ellipses(seed), W0, P0, axis=255.5)
    c0, outs0 = {}, {}
    for name, storage in (("plain_fp32", ufob.F32), ("fp16_storage", ufob.F16)):
        fbp = ufob.FBP(bp_props={"axis_pos": 255.5}, storage=storage)
        img = fbp.process(sino0)
        ms = _event_ms(torch, lambda: fbp.process(sino0, out=img), 200)
        c0[name] = {"us_per_slice": round(ms * 1e3, 2), "gups": round(W0 * W0 * P0 / ms / 1e6, 1)}
        outs0[name] = img.double().cpu().numpy()
    table["c0_single_slice"] = dict(workload="fft ! filter ! ifft ! backproject of one 512 px x 512 angle "
                                             "sinogram (10 random ellipses), axis 255.5, per call", **c0)
    checks["c0"] = (sino0.cpu().numpy(), outs0)
    del sino0

    # configuration 2: general-backproject, 1024 projections of 1024^2 over 360 degrees -> 512^3
    n_proj, det, vol = 1024, 1024, 512
    gen = torch.Generator(device=dev).manual_seed(seed)
    proj = torch.rand(n_proj, det, det, device=dev, generator=gen)
    h, q = vol / 2.0, 64
    base = {"center-position-x": det / 2.0, "center-position-z": det / 2.0,
            "x-region": (-h, h, 1.0), "y-region": (-h, h, 1.0), "region": (-h, h, 1.0)}
    c2, rois2 = {}, {}
    for gname, geom in C2_GEOMETRIES.items():
        # float: TMA-staged detector windows (the default); float_texture: the texture-gather
        # kernel; half: FP16 samples through texture gathers
        for form, ct, staging in (("float", "float", "auto"), ("float_texture", "float", "texture"),
                                  ("half", "half", "auto")):
            t = ufob.GeneralBackprojectTask(num_projections=n_proj)
            t.set_property("compute-type", ct)
            t.set_property("staging", staging)
            for k, v in list(base.items()) + list(geom.items()):
                t.set_property(k, v)
            v = t.process(proj)
            ms = _event_ms(torch, lambda: t.process(proj, out=v), 2)
            key = "%s_%s" % (gname, form)
            c2[key] = {"ms": round(ms, 2), "gups": round(float(vol) ** 3 * n_proj / ms / 1e6, 1)}
            rois2[key] = v[vol // 2, vol // 2 - q:vol // 2 + q, vol // 2 - q:vol // 2 + q].double().cpu().numpy()
            del t, v
    table["c2_general_backproject"] = dict(
        workload="general-backproject, %d projections of %d^2 over 360 degrees -> %d^3 (seeded uniform random "
                 "projections; the rate does not depend on the values), exact FP32 interpolation weights; "
                 "compute-type float with TMA-staged detector windows (default) and with texture gathers, "
                 "compute-type half (FP16 samples, FP32 arithmetic)" % (n_proj, det, vol), **c2)
    checks["c2"] = (proj.cpu().numpy(), base, q, rois2)
    del proj
    torch.cuda.empty_cache()

    # configuration 3: 64 uneven parallel-beam jobs in one persistent graph-captured launch pair
    rng = np.random.default_rng(seed)
    jobs, upd = [], 0
    for j in range(64):
        W = int(rng.choice([256, 512, 1024, 1536, 2048]))
        P = int(rng.integers(180, 1801))
        jobs.append(dict(sino=ufob.phantom_sinogram(random_ellipses(seed * 1000 + j), W, P),
                         out=torch.empty((W, W), device=dev)))
        upd += W * W * P
    c3, outs3 = {}, {}
    sizes = [j["sino"].shape[-1] ** 2 * j["sino"].shape[-2] for j in jobs]
    i_small, i_big = int(np.argmin(sizes)), int(np.argmax(sizes))
    i_1536 = next((i for i, j in enumerate(jobs) if j["sino"].shape[-1] == 1536), i_big)
    picks = sorted({i_small, i_big, i_1536})
    # checked region of each picked job: the whole slice up to 256^2, else the 128^2 block (on a
    # 64-pixel grid) with the most energy in a first FP32 run, so that an empty patch of the
    # phantom cannot inflate the relative error
    ufob.Batch(storage=ufob.F32).run(jobs)
    rois3 = []
    for i in picks:
        W = jobs[i]["sino"].shape[-1]
        if W <= 256:
            rois3.append((0, 0, W))
            continue
        img = jobs[i]["out"]
        e = torch.nn.functional.avg_pool2d((img * img)[None, None], 128, stride=64)[0, 0]
        k = int(torch.argmax(e))
        rois3.append(((k % e.shape[1]) * 64, (k // e.shape[1]) * 64, 128))
    for name, storage in (("fp32", ufob.F32), ("fp16", ufob.F16), ("bf16", ufob.BF16)):
        b = ufob.Batch(storage=storage)
        ms = _event_ms(torch, lambda: b.run(jobs), 3)
        c3[name] = {"ms": round(ms, 2), "gups": round(upd / ms / 1e6, 1), "tile_variant": b.variant()}
        outs3[name] = [jobs[i]["out"][y:y + n, x:x + n].double().cpu().numpy()
                       for i, (x, y, n) in zip(picks, rois3)]
        del b
    table["c3_uneven_batch"] = dict(workload="64 parallel-beam jobs, widths from {256,512,1024,1536,2048}, 180-1800 "
                                             "angles (seed %d), random-ellipse phantoms, %.3e updates" % (seed, upd),
                                    **c3)
    checks["c3"] = ([jobs[i]["sino"].cpu().numpy() for i in picks], rois3, outs3)
    del jobs
    torch.cuda.empty_cache()

    # configuration 4: learned 90-angle path (shipped weights) against dense 1800-angle FBP
    maker = PairMaker()
    net = SparseViewNet.pretrained()
    seeds = list(range(1_000_000, 1_000_064))
    imgs = maker.phantoms(seeds)
    s_sparse = maker.sinograms(imgs, maker.sparse)
    x = maker.fbp_sparse.process(s_sparse)
    x16 = ufob.FBP(storage=ufob.F16).process(s_sparse)
    y = maker.fbp_dense.process(maker.sinograms(imgs, maker.dense))
    times = [time_paths(net, maker, B=b) for b in (64, 128, 256)]
    table["c4_learned_sparse_view"] = {
        "workload": "90-angle 512 px FBP + 4-level CNN (32/64/128/256 ch, BF16 tensor cores) vs 1800-angle FBP, "
                    "shipped weights, 64 held-out phantoms (seeds 1e6..)",
        "plain_fbp90_rel_l2_vs_1800": round(float(rel_l2(x, y).mean()), 5),
        "cnn_rel_l2_vs_1800": round(float(rel_l2(net.forward(x), y).mean()), 5),
        "cnn_on_fp16_fbp90_rel_l2_vs_1800": round(float(rel_l2(net.forward(x16), y).mean()), 5),
        # the engine's learned path (FP16-storage 90-angle FBP + network) against the plain FP32
        # dense FBP, per batch size; the per-form ratios are under time_per_slice
        "learned_path_speedup_vs_plain_dense": {str(t["batch"]): t["fp16_learned_vs_plain_dense"] for t in times},
        "time_per_slice": times}
    del imgs, s_sparse, x, x16, y, net, maker
    torch.cuda.empty_cache()
    return table, checks


def config_errors(checks):
    """CPU leg of the other workloads: relative L2 errors of the sampled GPU outputs
    against the FP64 oracle and, for the one-slice FBP, the reference's own CPU build."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import reference
    err = {}
    sino0, outs0 = checks["c0"]
    ref64 = oracle.fbp(sino0, axis_pos=255.5)
    err["c0_single_slice"] = {k: {"rel_l2_vs_fp64": oracle.rel_l2(v, ref64)} for k, v in outs0.items()}
    if reference.available():
        refc = reference.backproject(reference.fft_filter_ifft(sino0).astype(np.float32), axis_pos=255.5)
        for k, v in outs0.items():
            err["c0_single_slice"][k]["rel_l2_vs_reference"] = oracle.rel_l2(v, refc)
    proj, base, q, rois2 = checks["c2"]
    err["c2_general_backproject"] = {}
    for gname, geom in C2_GEOMETRIES.items():
        kw = {k: v for k, v in list(base.items()) + list(geom.items()) if "region" not in k}
        ref = oracle.general_backproject(proj, proj.shape[0], region=(0.0, 1.0, 1.0), x_region=(-q, q, 1.0),
                                         y_region=(-q, q, 1.0), **kw)[0]
        for form in ("float", "float_texture", "half"):
            err["c2_general_backproject"]["%s_%s" % (gname, form)] = {
                "rel_l2_vs_fp64": oracle.rel_l2(rois2["%s_%s" % (gname, form)], ref),
                "sample": "central slice, %dx%d voxels" % (2 * q, 2 * q)}
    sinos3, rois3, outs3 = checks["c3"]
    refs3 = []
    for s, (x, y, n) in zip(sinos3, rois3):
        W = s.shape[-1]
        N = 1 << (W - 1).bit_length()
        refs3.append(oracle.backproject(oracle.fft_filter_ifft(s, size_x=N, crop_width=W).astype(np.float32),
                                        roi_x=x, roi_y=y, roi_width=n, roi_height=n))
    err["c3_uneven_batch"] = {k: {"rel_l2_vs_fp64_max": max(oracle.rel_l2(a, b) for a, b in zip(v, refs3)),
                                  "sample": "jobs (angles, width) %s, regions (x, y, side) %s"
                                            % ([tuple(s.shape) for s in sinos3], rois3)}
                              for k, v in outs3.items()}
    return err


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import numpy as np
    import torch
    import ufob

    from ufob import dist as udist
    # one process per GPU (torchrun env), independent slices per rank, NCCL only for the timing reductions
    ctx = udist.init(timeout_s=600)
    world, rank, dev = ctx.world, ctx.rank, ctx.device
    barrier, max_over_ranks = ctx.barrier, ctx.max_over_ranks

    Z, P, W = args.slices, args.angles, args.width
    updates_per_step = float(Z) * W * W * P
    smem_gbs, fp32_tflops = ufob.measure_peaks()
    stack = make_stack(ufob, torch, Z, P, W, args.seed + rank, dev)
    vol = torch.empty((Z, W, W), dtype=torch.float32, device=dev)

    # sampled slices / ROI for the FP64 error check
    rng = np.random.default_rng(args.seed)
    slice_ids = sorted(rng.choice(Z, size=min(4, Z), replace=False).tolist())
    side = min(256, W)
    if W >= 2 * side:
        rx, ry = [int(v) for v in rng.integers(W // 4, 3 * W // 4 - side // 2, size=2)]
    else:
        rx = ry = 0
    roi = (rx, ry, side, side)

    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    forms = {}
    launches_before = ufob.launch_count()
    total_launches = 0
    clocks_all = []
    for name, storage in (("plain_fp32", ufob.F32), ("fp16_storage", ufob.F16)):
        fbp = ufob.FBP(bp_props={"axis_pos": W / 2.0}, storage=storage)
        for _ in range(args.warmup):
            fbp.process(stack, out=vol)
        torch.cuda.synchronize()
        fbp.set_timing(True)
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(gpu_id)
        sampler.start()
        l0 = ufob.launch_count()
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fbp.process(stack, out=vol)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop()
        clocks_all.append(clocks)
        launches = ufob.launch_count() - l0
        total_launches += launches
        ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
        kt = fbp.kernel_times()
        fbp.set_timing(False)
        ufob.device_status()
        gpu_rois = vol[slice_ids, ry:ry + side, rx:rx + side].double().cpu().numpy()
        forms[name] = {"ms_per_step": ms, "gups": updates_per_step * world / (ms * 1e-3) / 1e9,
                       "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kt.items()},
                       "kernel_launches_per_step": {k: v[1] / args.steps for k, v in kt.items()},
                       "launches_per_step": launches / args.steps, "_rois": gpu_rois, "clocks": clocks}
        del fbp

    # CPU leg: oracle timing on a bounded sample + FP64 error reference (rank 0 only)
    cpu = None
    if rank == 0:
        host_slices = [stack[i].cpu().numpy() for i in slice_ids]
        cpu, errs = cpu_leg(host_slices, slice_ids, roi, P, W, {k: v["_rois"] for k, v in forms.items()})
        for k in forms:
            forms[k].update(errs[k])
    for k in forms:
        forms[k].pop("_rois")

    plain, fast = forms["plain_fp32"], forms["fp16_storage"]
    # the error is measured on rank 0 only: every rank takes rank 0's choice (the e2e leg must run the same form)
    fast_ok = 1.0 if (rank == 0 and fast.get("rel_l2_vs_fp64", 1.0) <= 1e-3 and fast["gups"] > plain["gups"]) else 0.0
    chosen_name = "fp16_storage" if ctx.sum_over_ranks(fast_ok) > 0.5 else "plain_fp32"
    chosen = forms[chosen_name]
    storage = ufob.F16 if chosen_name == "fp16_storage" else ufob.F32

    # end to end through the public host-pointer API (pinned host buffers, copies in the timed region)
    e2e = None
    if not args.no_e2e:
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 64 << 30
        per_slice = P * W * 4 + W * W * 4
        nz_e2e = args.e2e_slices or min(Z, max(8, int(0.35 * avail / world / per_slice) // 8 * 8))
        nz_e2e = min(nz_e2e, Z)
        h_in = torch.empty((nz_e2e, P, W), dtype=torch.float32, pin_memory=True)
        h_in.copy_(stack[:nz_e2e])
        h_out = torch.empty((nz_e2e, W, W), dtype=torch.float32, pin_memory=True)
        stack = vol = None
        torch.cuda.empty_cache()
        fbp = ufob.FBP(bp_props={"axis_pos": W / 2.0}, storage=storage)
        fbp.process_host(h_in[:min(16, nz_e2e)], out=h_out[:min(16, nz_e2e)], slices_per_chunk=16)
        times = []
        for i in range(args.steps):
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fbp.process_host(h_in, out=h_out, slices_per_chunk=64)
            torch.cuda.synchronize()
            times.append(max_over_ranks(time.perf_counter() - t0))
        dt = statistics.mean(times)
        e2e = {"value": nz_e2e * float(W) * W * P * world / dt / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": nz_e2e * P * W * 4, "d2h_bytes_per_step": nz_e2e * W * W * 4,
               "slices": nz_e2e, "s_per_step": dt,
               "api": "ufob_fbp_run_host (C ABI), pinned host buffers, 64-slice chunks (16-slice first and last) on two streams"}
        del fbp, h_in, h_out

    # the other four workloads (one-GPU configurations), timed on this GPU after the main arm, with
    # their own clock record; errors from the CPU leg
    configs = None
    if world == 1 and not args.no_configs:
        stack = vol = None
        torch.cuda.empty_cache()
        sampler = ClockSampler(gpu_id)
        sampler.start()
        table, checks = run_configs(ufob, torch, dev, args.seed)
        table["clocks"] = sampler.stop()
        ufob.device_status()
        for k, v in config_errors(checks).items():
            for form, e in v.items():
                table[k][form].update(e)
        configs = table

    # roofline of the dominant kernel (backprojection)
    bp_ms, bp_n = chosen["kernel_ms_per_step"]["backproject"], chosen["kernel_launches_per_step"]["backproject"]
    # on-chip bytes per update: 2 FP32 taps / one FP16 tap pair (a 16-byte cell serves 4 slices)
    gather_bytes = 8.0 if storage == ufob.F32 else 4.0
    upd_per_launch = updates_per_step / bp_n
    avg_launch_s = bp_ms / bp_n * 1e-3
    achieved = upd_per_launch * gather_bytes / avg_launch_s / 1e9
    bp_kernel = "k_bp_linear" if storage == ufob.F32 else "k_bp_quads"
    traffic_per_upd = read_profile_traffic("bp_linear_c1.md" if storage == ufob.F32 else "bp_quads_c1.md")
    roofline = {"bound": "smem", "kernel": bp_kernel, "achieved": achieved, "peak": smem_gbs, "unit": "GB/s",
                "frac": achieved / smem_gbs,
                "traffic": traffic_per_upd * upd_per_launch if traffic_per_upd is not None else None,
                "algorithmic_bytes_per_update": gather_bytes,
                "peak_source": "measured on this GPU by ufob_measure_peaks (32-bit shared loads); MEASURED_PEAKS.json "
                               "has no shared-memory figure",
                "gups_achieved_kernel": upd_per_launch / avg_launch_s / 1e9,
                "gups_roofline": smem_gbs / gather_bytes,
                "fp32_tflops_measured": fp32_tflops}
    # independent cross-check of the measured peak: 128 bytes per SM per clock (one shared-memory
    # wavefront) at the median SM clock sampled during the timed region
    sm_mhz = chosen["clocks"].get("sm_mhz")
    if sm_mhz:
        nominal = torch.cuda.get_device_properties(dev).multi_processor_count * 128.0 * sm_mhz * 1e6 / 1e9
        roofline["peak_nominal_gbs"] = nominal
        roofline["frac_of_nominal"] = achieved / nominal
    # the pool's measured copy bandwidth when the file is there, else the earlier pool measurement
    hbm_peak, hbm_source = HBM_FALLBACK_GBS, "fallback: 6.65 TB/s measured earlier on this pool (MEASURED_PEAKS.json absent)"
    try:
        hbm_peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
        hbm_source = "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError, TypeError):
        pass
    f_ms, f_n = chosen["kernel_ms_per_step"]["filter"], chosen["kernel_launches_per_step"]["filter"]
    f_bytes = Z * P * W * 4.0 + Z * P * (W if storage == ufob.F32 else (W + 1)) * 4.0
    f_kernel = "k_filter_fast" if 256 <= W <= 4096 and os.environ.get("UFOB_FILTER_RADIX4") != "1" else "k_filter_rows"
    roofline_filter = {"bound": "hbm", "kernel": f_kernel, "achieved": f_bytes / (f_ms * 1e-3) / 1e9,
                       "peak": hbm_peak, "unit": "GB/s",
                       "frac": (f_bytes / (f_ms * 1e-3) / 1e9) / hbm_peak,
                       "peak_source": hbm_source}

    clk = dict(chosen["clocks"])
    if rank == 0:
        line = {
            "metric": METRIC, "value": chosen["gups"], "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": chosen["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if storage == ufob.F32 else "f32 accumulate, f16 filtered-sinogram storage",
            "data": "synthetic: 50 random ellipsoids, analytic line integrals, Beer-Lambert I0=1e4 + Poisson noise",
            "config": {"workload": WORKLOAD, "slices_per_gpu": Z, "width": W, "angles": P,
                       "chosen_form": chosen_name, "parallelism": "independent slices per GPU" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (%.1f GB sinogram stack per GPU)" % (Z * P * W * 4 / 1e9),
                       "error_sample": "slices %s, ROI x=%d y=%d %dx%d" % (slice_ids, rx, ry, side, side)},
            "forms": forms,
            "roofline": roofline,
            "roofline_filter": roofline_filter,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(round(chosen["launches_per_step"] * args.steps)),
            "clocks": clk,
            "configs": configs,
        }
        print(json.dumps(line), flush=True)
    udist.finish(ctx)


if __name__ == "__main__":
    main()
