"""Multi-GPU plumbing: one process per GPU, independent slices per rank.

Parallel-beam slices are independent, so a stack is split into contiguous
slice ranges, one per rank, and every rank reconstructs its own range with no
collective in the data path.  The only collectives are the timing reductions
(max over ranks) and, if the caller wants one volume on one host, a gather of
the reconstructed slices to rank 0 at the end.  Rank/world come from the
torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT); the
backend is NCCL when CUDA is available and gloo otherwise (CPU tests).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ctx:
    rank: int = 0
    world: int = 1
    local: int = 0
    device: object = None
    group: object = None  # torch.distributed module when world > 1

    def barrier(self):
        if self.group is not None:
            self.group.barrier()

    def _reduce(self, x, op):
        if self.group is None:
            return x
        import torch
        dev = self.device if self.group.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.group.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(self, x):
        return self._reduce(x, None if self.group is None else self.group.ReduceOp.MAX)

    def sum_over_ranks(self, x):
        return self._reduce(x, None if self.group is None else self.group.ReduceOp.SUM)


def init(backend=None, timeout_s=600):
    """Join the process group described by the environment (no-op for one process)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cuda = torch.cuda.is_available()
    dev = torch.device("cuda", local) if cuda else torch.device("cpu")
    if cuda:
        torch.cuda.set_device(local)
    ctx = Ctx(rank=rank, world=world, local=local, device=dev)
    if world > 1:
        import torch.distributed as dist
        backend = backend or ("nccl" if cuda else "gloo")
        kw = {"device_id": dev} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), rank=rank, world_size=world,
                                **kw)
        ctx.group = dist
    return ctx


def finish(ctx):
    if ctx.group is not None:
        ctx.group.destroy_process_group()
        ctx.group = None


def slice_range(n, rank, world):
    """Contiguous, balanced [start, stop) share of n slices for one rank."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def reconstruct_sharded(ctx, stack, reconstruct, gather=False):
    """Reconstruct this rank's slice range of `stack` ([Z, P, W], host or
    device) with `reconstruct(sub_stack) -> sub_volume` (CPU torch tensor or
    numpy array).  Returns (start, stop, local volume); with `gather`, rank 0
    receives the whole volume instead (other ranks get None)."""
    import numpy as np
    import torch
    start, stop = slice_range(stack.shape[0], ctx.rank, ctx.world)
    local = reconstruct(stack[start:stop])
    if not gather or ctx.group is None:
        return start, stop, local
    # point-to-point transfers run on the device for NCCL and on the host for gloo
    dev = ctx.device if ctx.group.get_backend() == "nccl" else "cpu"
    t = torch.as_tensor(np.asarray(local) if not torch.is_tensor(local) else local).contiguous().to(dev)
    shapes = [None] * ctx.world
    ctx.group.all_gather_object(shapes, tuple(t.shape))
    if ctx.rank == 0:
        parts = [t] + [torch.empty(s, dtype=t.dtype, device=dev) for s in shapes[1:]]
        for r in range(1, ctx.world):
            ctx.group.recv(parts[r], src=r)
        return 0, stack.shape[0], torch.cat(parts).cpu()
    ctx.group.send(t, dst=0)
    return start, stop, None
