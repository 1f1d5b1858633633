"""Multi-GPU layout of the DD path: one process per GPU.

Two ways to spread the work, matching how the path partitions:

* independent problems (batch members, instances) run as replicas, one
  share per rank, with no collective on the data path (``batch_shard``);
* one large 3D problem is split inside:
  - the projection A by views: every rank projects the whole volume for its
    own views (``view_shard``); no exchange;
  - the backprojection B / Bw (and the voxel-owned A^T) by z-slabs of the
    volume: each rank needs every view, so the view-sharded sinogram is
    all-gathered once (one ``all_gather`` over NCCL / NVLink), then each
    rank backprojects its own slab.  A slab is itself a volume geometry (``slab_options``), so the
    voxel-owned backprojection of the slab equals the slab of the full
    backprojection.

The operators are passed in as callables ``op(x, options, angles)`` (the
``xrecon_b200.backend`` functions on GPU), which keeps this module free of
device code.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch
import torch.distributed as dist


def _split(n: int, rank: int, world: int) -> slice:
    """Contiguous share of ``n`` items for ``rank``; the first ``n % world``
    ranks get one more."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def batch_shard(n: int, rank: int, world: int) -> slice:
    """Batch members (or instances) of one rank."""
    return _split(n, rank, world)


def view_shard(nview: int, rank: int, world: int) -> slice:
    """Views of one rank for the view-sharded projection."""
    return _split(nview, rank, world)


def slab_shard(depth: int, rank: int, world: int) -> slice:
    """z-slices of one rank for the slab-sharded backprojection."""
    return _split(depth, rank, world)


def slab_options(options: Sequence[float], zs: slice) -> list:
    """Packed 3D options (the 18 values of ``pack_options3d``) of the slab
    ``zs`` of the volume: depth ``zs.stop - zs.start`` and the z shift that
    puts its voxels where they are in the full volume.  z boundaries are
    ``-D dz / 2 + shift_z + k dz`` (torch_binding.cpp:82-124 unpacking)."""
    o = [float(v) for v in options]
    D, dz, shz = int(o[2]), o[7], o[14]
    start, stop = zs.start or 0, D if zs.stop is None else zs.stop
    if not (0 <= start < stop <= D):
        raise ValueError(f"slab {start}:{stop} outside depth {D}")
    d = stop - start
    o[2] = float(d)
    o[14] = shz + (start + 0.5 * d - 0.5 * D) * dz
    return o


def project_views(op: Callable, vol: torch.Tensor, options, angles: torch.Tensor, rank: int,
                  world: int) -> torch.Tensor:
    """This rank's views of A(vol): [B, C, V_rank, Nv, Nu]."""
    vs = view_shard(angles.numel(), rank, world)
    return op(vol, options, angles[vs].contiguous())


def gather_views(sino_local: torch.Tensor, nview: int, group=None) -> torch.Tensor:
    """All-gather view shards (as produced by ``project_views``) into the
    full sinogram [B, C, V, ...] on every rank.

    One all-gather of equal-sized buffers: when the views do not split
    evenly, every shard is padded to the largest one and trimmed after the
    exchange (collectives such as gloo's all-gather need equal sizes)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = [view_shard(nview, r, world) for r in range(world)]
    counts = [vs.stop - vs.start for vs in counts]
    if sino_local.shape[2] != counts[rank]:
        raise ValueError(f"rank {rank} holds {sino_local.shape[2]} views, its shard has {counts[rank]}")
    vmax = max(counts)
    shape = (sino_local.shape[0], sino_local.shape[1], vmax) + tuple(sino_local.shape[3:])
    send = sino_local.contiguous()
    if counts[rank] != vmax:
        send = torch.zeros(shape, dtype=sino_local.dtype, device=sino_local.device)
        send[:, :, :counts[rank]] = sino_local
    bufs = [torch.empty(shape, dtype=sino_local.dtype, device=sino_local.device) for _ in range(world)]
    dist.all_gather(bufs, send, group=group)
    return torch.cat([b[:, :, :n] for b, n in zip(bufs, counts)], dim=2)


def backproject_slab(op: Callable, sino: torch.Tensor, options, angles: torch.Tensor, rank: int,
                     world: int) -> tuple[slice, torch.Tensor]:
    """This rank's z-slab of ``op`` (B, Bw or A^T: the voxel-owned
    operators) applied to the full sinogram:
    (slab slice, [B, C, D_rank, H, W]).  With more ranks than slices, a rank
    without slices gets an empty slab and ``op`` is not called."""
    D = int(float(options[2]))
    zs = slab_shard(D, rank, world)
    if zs.stop == zs.start:
        H, W = int(float(options[1])), int(float(options[0]))
        return zs, torch.zeros((sino.shape[0], sino.shape[1], 0, H, W), dtype=sino.dtype, device=sino.device)
    opts = slab_options(options, zs)
    if isinstance(options, torch.Tensor):
        opts = torch.tensor(opts, dtype=options.dtype, device=options.device)
    return zs, op(sino, opts, angles)


def max_over_ranks(seconds: float, device=None, group=None) -> float:
    """The slowest rank's time (the job's time) for a per-rank measurement."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return seconds
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sharded_projection_backprojection(fwd: Callable, back: Callable, vol: torch.Tensor, options,
                                      angles: torch.Tensor, rank: int, world: int, group=None,
                                      marks: Callable | None = None) -> tuple[slice, torch.Tensor]:
    """One A-then-B step of a single problem split over the ranks: this
    rank's views of A(vol), the view shards all-gathered (one collective),
    then this rank's z-slab of B applied to the full sinogram.  Returns
    (slab slice, slab of B(A(vol))).  ``vol`` is the full volume on every
    rank.  ``marks(name)``, when given, is called after each phase
    ("projection", "gather", "backprojection") so a caller can time them on
    its stream."""
    local = project_views(fwd, vol, options, angles, rank, world)
    if marks:
        marks("projection")
    full = gather_views(local, angles.numel(), group) if world > 1 else local
    if marks:
        marks("gather")
    zs, slab = backproject_slab(back, full, options, angles, rank, world)
    if marks:
        marks("backprojection")
    return zs, slab
