"""Train and evaluate the 90-angle sparse-view correction network.

    python -m ufob.train_cnn --pairs 20000 --epochs 8 --ckpt cnn.npz
    python -m ufob.train_cnn --pretrained          # evaluate and time the shipped weights

Pairs (90-angle FBP, 1800-angle FBP) of seeded random-ellipse phantoms at
512^2 are made on the GPU by the engine's own projector and FBP and cached in
device memory (20k pairs are 42 GB); training takes Adam steps over shuffled
mini-batches with a cosine learning-rate schedule and checkpoints to .npz
(resumable).  Evaluation uses a disjoint seed range and reports the mean
relative L2 error against the 1800-angle FBP of plain 90-angle FBP and of
FBP + network, and the batched time per slice of the learned path against a
dense 1800-angle FBP.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np


def make_cache(maker, seeds, batch=32):
    import torch
    xs, ys = [], []
    for i in range(0, len(seeds), batch):
        x, y, _ = maker.pair(seeds[i:i + batch])
        xs.append(x)
        ys.append(y)
    torch.cuda.synchronize()
    return torch.cat(xs), torch.cat(ys)


def time_paths(net, maker, B=64, reps=5):
    """Batched time per slice: sparse FBP + network vs dense FBP (FP32 and FP16-storage FBP)."""
    import torch
    from . import F16, F32, FBP
    imgs = maker.phantoms(list(range(10**7, 10**7 + B)))
    s_sparse = maker.sinograms(imgs, maker.sparse)
    s_dense = maker.sinograms(imgs, maker.dense)

    def t(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(True), torch.cuda.Event(True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps * 1e3 / B  # us per slice

    out = {"batch": B}
    for name, storage in (("fp32", F32), ("fp16", F16)):
        fbp = FBP(storage=storage)
        x = fbp.process(s_sparse)
        t_sparse = t(lambda: fbp.process(s_sparse))
        t_dense = t(lambda: fbp.process(s_dense))
        t_net = t(lambda: net.forward(x))
        t_learned = t(lambda: net.forward(fbp.process(s_sparse)))
        out[name] = {"sparse_fbp_us": round(t_sparse, 2), "network_us": round(t_net, 2),
                     "learned_path_us": round(t_learned, 2), "dense_fbp_us": round(t_dense, 2),
                     "speedup_vs_dense": round(t_dense / t_learned, 2)}
    # the engine's fastest learned path (FP16-storage sparse FBP + network) against the plain dense FBP
    out["fp16_learned_vs_plain_dense"] = round(out["fp32"]["dense_fbp_us"] / out["fp16"]["learned_path_us"], 2)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--epochs", type=float, default=8)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed-base", type=int, default=0)
    ap.add_argument("--eval-base", type=int, default=1_000_000)
    ap.add_argument("--eval-count", type=int, default=256)
    ap.add_argument("--ckpt", default="")
    ap.add_argument("--ckpt-every", type=int, default=1000)
    ap.add_argument("--log-every", type=int, default=250)
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--pretrained", action="store_true", help="evaluate the shipped weights (implies --eval-only)")
    ap.add_argument("--time-batches", default="64,128,256", help="batch sizes of the timing comparison")
    args = ap.parse_args(argv)

    import torch
    from .cnn import PairMaker, SparseViewNet, rel_l2

    maker = PairMaker()
    start = 0
    if args.pretrained:
        net = SparseViewNet.pretrained()
        args.eval_only = True
    else:
        net = SparseViewNet(seed=1234)
        if args.ckpt and os.path.exists(args.ckpt):
            start = int(net.load(args.ckpt).get("train_step", 0))
    steps = int(math.ceil(args.epochs * args.pairs / args.batch))
    report = {"pairs": args.pairs, "batch": args.batch, "steps": steps, "resumed_at": start}
    t0 = time.time()
    if not args.eval_only and start < steps:
        X, Y = make_cache(maker, list(range(args.seed_base, args.seed_base + args.pairs)))
        report["pair_generation_s"] = round(time.time() - t0, 1)
        rng = np.random.default_rng(args.seed_base + 7)
        perm, losses = [], []
        t1 = time.time()
        for it in range(steps):
            if not perm:
                perm = list(rng.permutation(args.pairs))
            idx = [perm.pop() for _ in range(min(args.batch, len(perm)))]
            if it < start:
                continue  # replay the shuffle stream up to the checkpoint
            sel = torch.tensor(idx, device=X.device)
            lr = 1e-5 + 0.5 * (args.lr - 1e-5) * (1 + math.cos(math.pi * it / steps))
            losses.append(net.train_step(X.index_select(0, sel), Y.index_select(0, sel), lr))
            if args.log_every and (it + 1) % args.log_every == 0:
                print(f"step {it + 1}/{steps} loss {np.mean(losses[-args.log_every:]):.4e} lr {lr:.2e}",
                      file=sys.stderr, flush=True)
            if args.ckpt and (it + 1) % args.ckpt_every == 0:
                net.save(args.ckpt, train_step=it + 1)
        report["train_s"] = round(time.time() - t1, 1)
        report["final_loss"] = float(np.mean(losses[-200:])) if losses else None
        del X, Y
        if args.ckpt:
            net.save(args.ckpt, train_step=steps)
    from . import F16, FBP
    fbp16 = FBP(storage=F16)
    e_plain, e_net, e_net16 = [], [], []
    eval_seeds = list(range(args.eval_base, args.eval_base + args.eval_count))
    for i in range(0, len(eval_seeds), 32):
        imgs = maker.phantoms(eval_seeds[i:i + 32])
        s_sparse = maker.sinograms(imgs, maker.sparse)
        x = maker.fbp_sparse.process(s_sparse)
        y = maker.fbp_dense.process(maker.sinograms(imgs, maker.dense))
        e_plain.append(rel_l2(x, y))
        e_net.append(rel_l2(net.forward(x), y))
        e_net16.append(rel_l2(net.forward(fbp16.process(s_sparse)), y))
    report["eval"] = {"seeds": [args.eval_base, args.eval_base + args.eval_count],
                      "plain_fbp90_rel_l2": round(float(torch.cat(e_plain).mean()), 5),
                      "cnn_rel_l2": round(float(torch.cat(e_net).mean()), 5),
                      "cnn_on_fp16_fbp90_rel_l2": round(float(torch.cat(e_net16).mean()), 5)}
    report["time_per_slice"] = [time_paths(net, maker, B=int(b)) for b in args.time_batches.split(",")]
    print(json.dumps(report))


if __name__ == "__main__":
    main()
