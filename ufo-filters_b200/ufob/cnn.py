"""Learned 90-angle sparse-view correction.

A small U-Net (4 levels, 32/64/128/256 channels, 3x3 convolutions, BF16
weights and activations, FP32 accumulation on the tcgen05 tensor cores) maps
the FBP of a 90-angle sinogram to a correction added to it.  It is trained
only on pairs the engine makes itself: random ellipse phantoms rasterised on
the GPU, forward-projected with the engine's projector over 90 and 1800
angles, and reconstructed with the engine's FBP; the target is the
1800-angle FBP.  Plain FBP stays the fallback and the judge of the error.

All compute runs in libufob (cnn_net.cu, cnn_conv.cu for training, cnn_fast.cu
for inference); this module holds the
data generation loop, checkpointing and evaluation.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from . import FBP, _ptr, _stream, check, forwardproject, lib, phantom_images

PARAMS, GRADS, ADAM_M, ADAM_V = 0, 1, 2, 3


def random_ellipses(seed, n=10):
    """Ellipse phantom rows (cx, cy, a, b, phi, rho): centres uniform in the
    unit disc, semi-axes U[0.05, 0.4], angle U[0, pi), density U[-0.5, 1]."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0, 1, n))
    t = rng.uniform(0, 2 * math.pi, n)
    out = np.empty((n, 6))
    out[:, 0] = r * np.cos(t)
    out[:, 1] = r * np.sin(t)
    out[:, 2] = rng.uniform(0.05, 0.4, n)
    out[:, 3] = rng.uniform(0.05, 0.4, n)
    out[:, 4] = rng.uniform(0, math.pi, n)
    out[:, 5] = rng.uniform(-0.5, 1.0, n)
    return out


class PairMaker:
    """Phantom -> (90-angle FBP, 1800-angle FBP) pairs, all on the GPU."""

    def __init__(self, N=512, sparse=90, dense=1800, phantom_scale=None):
        self.N, self.sparse, self.dense = N, sparse, dense
        # phantoms fill 90% of the reconstruction circle
        self.phantom_scale = phantom_scale or 0.45 * N
        self.fbp_sparse = FBP()
        self.fbp_dense = FBP()

    def phantoms(self, seeds):
        return phantom_images([random_ellipses(int(s)) for s in seeds], self.N, scale=self.phantom_scale)

    def sinograms(self, imgs, n_angles):
        import torch
        out = torch.empty((imgs.shape[0], n_angles, self.N), dtype=torch.float32, device=imgs.device)
        for i in range(imgs.shape[0]):
            forwardproject(imgs[i], n_angles, out=out[i])
        return out

    def pair(self, seeds):
        imgs = self.phantoms(seeds)
        x = self.fbp_sparse.process(self.sinograms(imgs, self.sparse))
        y = self.fbp_dense.process(self.sinograms(imgs, self.dense))
        return x, y, imgs


class SparseViewNet:
    """Handle on the engine's correction network (one per device)."""

    def __init__(self, seed=0, scale=1.0):
        h = ctypes.c_void_p()
        check(lib().ufob_cnn_create(seed, scale, ctypes.byref(h)))
        self._h = h
        self._destroy = lib().ufob_cnn_destroy  # bound now: module globals may be gone at exit
        self.scale = scale
        self.n_params = int(lib().ufob_cnn_num_params())

    @classmethod
    def pretrained(cls, path=None):
        """The network trained by `python -m ufob.train_cnn` (20k engine-made pairs,
        512^2, 90 -> 1800 angles), shipped as weights/sparse_view_90to1800_512.npz."""
        path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                    "sparse_view_90to1800_512.npz")
        d = np.load(path)
        net = cls(seed=0, scale=float(d["scale"]))
        net.set_state(PARAMS, d["params"])
        return net

    def forward(self, fbp, out=None, stream=None):
        """[B, H, W] FP32 CUDA tensor (sides multiples of 32) -> corrected slices."""
        import torch
        x = fbp.contiguous()
        B, H, W = x.shape
        out = torch.empty_like(x) if out is None else out
        check(lib().ufob_cnn_forward(self._h, _ptr(x), _ptr(out), B, H, W, _stream(stream)))
        return out

    def forward_nhwc(self, fbp, out=None, stream=None):
        """The same network through the training kernels (for checks)."""
        import torch
        x = fbp.contiguous()
        B, H, W = x.shape
        out = torch.empty_like(x) if out is None else out
        check(lib().ufob_cnn_forward_nhwc(self._h, _ptr(x), _ptr(out), B, H, W, _stream(stream)))
        return out

    def train_step(self, fbp, target, lr, stream=None):
        """One Adam step on the MSE between forward(fbp) and target; returns the loss."""
        loss = ctypes.c_double()
        x, y = fbp.contiguous(), target.contiguous()
        B, H, W = x.shape
        check(lib().ufob_cnn_train_step(self._h, _ptr(x), _ptr(y), B, H, W, float(lr), ctypes.byref(loss),
                                        _stream(stream)))
        return loss.value

    def get_state(self, which=PARAMS):
        out = np.empty(self.n_params, dtype=np.float32)
        check(lib().ufob_cnn_get_state(self._h, which, out.ctypes.data, out.size))
        return out

    def set_state(self, which, values):
        v = np.ascontiguousarray(values, dtype=np.float32)
        check(lib().ufob_cnn_set_state(self._h, which, v.ctypes.data, v.size))

    @property
    def step(self):
        return int(lib().ufob_cnn_get_step(self._h))

    def save(self, path, **extra):
        """Checkpoint parameters, Adam moments and step to an .npz file."""
        tmp = path + ".tmp.npz"
        np.savez(tmp, params=self.get_state(PARAMS), adam_m=self.get_state(ADAM_M),
                 adam_v=self.get_state(ADAM_V), step=self.step, scale=self.scale, **extra)
        os.replace(tmp, path)

    def load(self, path):
        """Resume from a checkpoint written by save(); returns its extra entries."""
        d = np.load(path)
        self.set_state(PARAMS, d["params"])
        self.set_state(ADAM_M, d["adam_m"])
        self.set_state(ADAM_V, d["adam_v"])
        check(lib().ufob_cnn_set_step(self._h, int(d["step"])))
        return {k: d[k] for k in d.files if k not in ("params", "adam_m", "adam_v", "step", "scale")}

    def __del__(self):
        h, fn = getattr(self, "_h", None), getattr(self, "_destroy", None)
        if h and fn:
            fn(h)
            self._h = None


def rel_l2(a, b):
    """Per-image relative L2 error of a against b (torch tensors [B, H, W])."""
    d = (a - b).flatten(1).norm(dim=1)
    return d / b.flatten(1).norm(dim=1).clamp_min(1e-30)


def train(steps, batch=16, lr=1e-3, seed_base=0, n_train=20000, ckpt=None, ckpt_every=500, log_every=100,
          net=None, maker=None, lr_final=1e-5, log=print):
    """Train on seeds [seed_base, seed_base + n_train): each step draws `batch`
    seeds, makes their pairs on the GPU and takes one Adam step; cosine
    learning-rate decay to lr_final.  Resumes from `ckpt` if it exists."""
    maker = maker or PairMaker()
    net = net or SparseViewNet(seed=1234)
    start = 0
    if ckpt and os.path.exists(ckpt):
        start = int(net.load(ckpt).get("train_step", 0))
    rng = np.random.default_rng(seed_base + 7)
    for _ in range(start):  # keep the seed stream identical across resumes
        rng.integers(0, n_train, batch)
    losses = []
    for it in range(start, steps):
        seeds = seed_base + rng.integers(0, n_train, batch)
        x, y, _ = maker.pair(seeds)
        cur = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * it / max(steps, 1)))
        losses.append(net.train_step(x, y, cur))
        if log and (it + 1) % log_every == 0:
            log(f"step {it + 1} loss {np.mean(losses[-log_every:]):.4e} lr {cur:.2e}")
        if ckpt and (it + 1) % ckpt_every == 0:
            net.save(ckpt, train_step=it + 1)
    if ckpt:
        net.save(ckpt, train_step=steps)
    return net, losses


def evaluate(net, seeds, maker=None, batch=16):
    """Mean relative L2 vs the 1800-angle FBP of plain 90-angle FBP and of
    FBP + network on held-out seeds."""
    import torch
    maker = maker or PairMaker()
    e_plain, e_net = [], []
    for i in range(0, len(seeds), batch):
        x, y, _ = maker.pair(seeds[i:i + batch])
        out = net.forward(x)
        e_plain.append(rel_l2(x, y))
        e_net.append(rel_l2(out, y))
    torch.cuda.synchronize()
    return float(torch.cat(e_plain).mean()), float(torch.cat(e_net).mean())


def _main(argv=None):
    """python -m ufob.cnn [--batch B] [--reps R]: time the inference path on
    B random 512^2 slices (the shipped weights), one JSON line."""
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args(argv)
    net = SparseViewNet.pretrained()
    x = torch.randn(args.batch, 512, 512, device="cuda") * 0.3
    net.forward(x)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.reps):
        net.forward(x)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.reps
    flop = 1.208e9 * args.batch  # sum over the 8 convolutions of 2 * 9 * Cin * Cout * H * W
    print(json.dumps({"workload": "sparse-view network forward, %d x 512^2" % args.batch, "ms": round(ms, 3),
                      "us_per_slice": round(ms * 1e3 / args.batch, 2), "tflops": round(flop / ms / 1e9, 1)}))


if __name__ == "__main__":
    _main()
