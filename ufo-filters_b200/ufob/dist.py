"""Multi-GPU plumbing: one process per GPU, independent slices per rank.

Parallel-beam slices are independent, so a stack is split into contiguous
slice ranges, one per rank, and every rank reconstructs its own range with no
collective in the data path.  The only collectives are the timing reductions
(max over ranks) and, if the caller wants one volume on one host, a gather of
the reconstructed slices to rank 0 at the end.

Cone-beam and laminography volumes (general-backproject) are partitioned
along z instead: every slice needs every projection, so each rank filters its
share of the projections, one all-gather gives every rank all filtered
projections, and each rank backprojects its own z range
(`reconstruct_volume_sharded`).  Rank/world come from the
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


def _all_gather_uneven(ctx, t, counts):
    """All-gather of rank shares along dim 0 with counts[r] rows from rank r
    (padded to the largest share for the collective); returns the concatenation."""
    import torch
    if ctx.group is None:
        return t
    mx = max(counts)
    pad = t if t.shape[0] == mx else torch.cat([t, t.new_zeros((mx - t.shape[0],) + tuple(t.shape[1:]))])
    parts = [torch.empty_like(pad) for _ in range(ctx.world)]
    ctx.group.all_gather(parts, pad.contiguous())
    return torch.cat([p[:c] for p, c in zip(parts, counts)])


def reconstruct_volume_sharded(ctx, proj_share, n_projections, z_region, filter_fn, backproject_fn, gather=False):
    """Filter this rank's share of the projections, exchange them, and backproject this
    rank's z range.

    proj_share: projections slice_range(n_projections, rank, world) of the stack
    ([n_r, H, W], device tensor with NCCL, CPU tensor with gloo); z_region: the whole
    volume's (from, to, step); filter_fn(projections) -> filtered projections;
    backproject_fn(all_filtered, (from, to, step)) -> volume [nz_r, ny, nx] of this
    rank's slices.  Returns (z0, z1, local volume); with `gather`, rank 0 receives the
    whole volume (others get None)."""
    import math
    import torch
    start, step = float(z_region[0]), float(z_region[2])
    nz = int(math.ceil((float(z_region[1]) - start) / step))
    counts = [b - a for a, b in (slice_range(n_projections, r, ctx.world) for r in range(ctx.world))]
    if proj_share.shape[0] != counts[ctx.rank]:
        raise ValueError("rank %d holds %d projections, expected %d" % (ctx.rank, proj_share.shape[0],
                                                                       counts[ctx.rank]))
    filtered = torch.as_tensor(filter_fn(proj_share))
    everything = _all_gather_uneven(ctx, filtered, counts)  # the one exchange step
    z0, z1 = slice_range(nz, ctx.rank, ctx.world)
    # this rank's slices: the same z values as the whole region's z0 .. z1 - 1
    local = backproject_fn(everything, (start + z0 * step, start + (z1 - 0.5) * step, step)) if z1 > z0 else None
    if not gather or ctx.group is None:
        return z0, z1, local
    dev = ctx.device if ctx.group.get_backend() == "nccl" else "cpu"
    t = torch.as_tensor(local).contiguous().to(dev) if local is not None else None
    shapes = [None] * ctx.world
    ctx.group.all_gather_object(shapes, tuple(t.shape) if t is not None else None)
    if ctx.rank == 0:
        parts = [t] if t is not None else []
        for r in range(1, ctx.world):
            if shapes[r] is None:
                continue
            buf = torch.empty(shapes[r], dtype=t.dtype if t is not None else torch.float32, device=dev)
            ctx.group.recv(buf, src=r)
            parts.append(buf)
        return 0, nz, torch.cat(parts).cpu()
    if t is not None:
        ctx.group.send(t, dst=0)
    return z0, z1, None
