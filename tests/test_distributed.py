"""Multi-rank host logic on CPU: gloo, world sizes 2 and 3, the FP64 oracle
as the operator.  View-sharded projection + all-gather + slab-sharded
backprojection equals the single-process result (with 3 ranks the 16 views
and 11 slices split unevenly); shards cover everything once; slab geometries reproduce the full volume's voxels (to the float32
rounding of the slab's z shift in the packed options, ~2e-7 relative)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_golden
from oracle import oracle as O
from xrecon_b200 import distributed as XD


@pytest.mark.parametrize("n,world", [(0, 1), (1, 2), (7, 2), (8, 3), (1440, 8), (5, 8)])
def test_shards_cover_each_item_once(n, world):
    seen = []
    for r in range(world):
        s = XD.view_shard(n, r, world)
        seen.extend(range(s.start, s.stop))
    assert seen == list(range(n))


def test_slab_options_reproduce_full_volume():
    g = load_golden("dd3d_flat")
    opts, ang = g["options"], g["angles"]
    sino = g["sino"]
    full = O.dd3d("B", sino, opts, ang)
    D = int(opts[2])
    parts = []
    for r in range(3):
        zs = XD.slab_shard(D, r, 3)
        parts.append(O.dd3d("BW" if r == 1 else "B", sino, XD.slab_options(opts, zs), ang))
    bw = O.dd3d("BW", sino, opts, ang)
    zs1 = XD.slab_shard(D, 1, 3)
    np.testing.assert_allclose(parts[1], bw[:, :, zs1], rtol=1e-6, atol=1e-6 * np.abs(bw).max())
    zs0, zs2 = XD.slab_shard(D, 0, 3), XD.slab_shard(D, 2, 3)
    np.testing.assert_allclose(parts[0], full[:, :, zs0], rtol=1e-6, atol=1e-6 * np.abs(full).max())
    np.testing.assert_allclose(parts[2], full[:, :, zs2], rtol=1e-6, atol=1e-6 * np.abs(full).max())


@pytest.mark.parametrize("geom", ["dd3d_flat", "dd3d_arc", "dd3d_parallel"])
def test_slab_options_serve_the_projection_transpose(geom):
    """A^T is voxel-owned like B, so the slab-sharded layout also serves it
    (the reduce-scatter of a view-sharded A^T is not needed)."""
    g = load_golden(geom)
    opts, ang, sino = g["options"], g["angles"], g["sino"]
    full = O.dd3d("AT", sino, opts, ang)
    D = int(opts[2])
    for r in range(3):
        zs = XD.slab_shard(D, r, 3)
        part = O.dd3d("AT", sino, XD.slab_options(opts, zs), ang)
        np.testing.assert_allclose(part, full[:, :, zs], rtol=1e-6, atol=1e-6 * np.abs(full).max())


def test_more_ranks_than_slices_leaves_empty_slabs():
    g = load_golden("dd3d_flat")
    opts, ang, sino = g["options"], torch.from_numpy(g["angles"]), torch.from_numpy(g["sino"])
    D, H, W = int(opts[2]), int(opts[1]), int(opts[0])
    world = D + 3
    calls = []

    def op(x, options, angles):
        calls.append(int(float(options[2])))
        return torch.zeros((x.shape[0], x.shape[1], int(float(options[2])), H, W))

    depth = 0
    for r in range(world):
        zs, slab = XD.backproject_slab(op, sino, opts, ang, r, world)
        assert slab.shape == (1, 1, zs.stop - zs.start, H, W)
        depth += slab.shape[2]
    assert depth == D and calls == [1] * D


def _oracle_op(name):
    def op(x, options, angles):
        o = np.asarray(options.tolist() if isinstance(options, torch.Tensor) else options, np.float32)
        return torch.from_numpy(O.dd3d(name, x.numpy(), o, angles.numpy()))
    return op


def _worker(rank, world, port, q, nview):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = load_golden("dd3d_arc")
        opts = torch.from_numpy(g["options"])
        ang = torch.from_numpy(g["angles"][:nview])
        vol = torch.from_numpy(g["image"]).double()
        local = XD.project_views(_oracle_op("A"), vol, opts, ang, rank, world)
        sino = XD.gather_views(local, ang.numel())
        zs, slab = XD.backproject_slab(_oracle_op("B"), sino, opts, ang, rank, world)
        t = XD.max_over_ranks(float(rank + 1))
        q.put((rank, zs.start, zs.stop, slab.numpy(), sino.numpy(), t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nview", [(2, 16), (3, 16), (3, 2)])
def test_view_and_slab_sharding_matches_single_process(world, nview):
    """2 ranks split evenly; 3 ranks split the 16 views and 11 slices
    unevenly; with 2 views one of the 3 ranks projects no view at all."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, nview)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = load_golden("dd3d_arc")
    ang = g["angles"][:nview]
    assert ang.size == nview
    sino_ref = O.dd3d("A", g["image"], g["options"], ang)
    vol_ref = O.dd3d("B", sino_ref, g["options"], ang)
    out = np.zeros_like(vol_ref)
    for rank, z0, z1, slab, sino, t in results:
        np.testing.assert_allclose(sino, sino_ref, rtol=1e-12, atol=1e-12 * np.abs(sino_ref).max())
        out[:, :, z0:z1] = slab
        assert t == float(world)  # max over ranks
    np.testing.assert_allclose(out, vol_ref, rtol=1e-6, atol=1e-6 * np.abs(vol_ref).max())


def _step_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = load_golden("dd3d_flat")
        opts = torch.from_numpy(g["options"])
        ang = torch.from_numpy(g["angles"])
        vol = torch.from_numpy(g["image"]).double()
        phases = []
        zs, slab = XD.sharded_projection_backprojection(_oracle_op("A"), _oracle_op("B"), vol, opts, ang, rank,
                                                        world, marks=phases.append)
        q.put((rank, zs.start, zs.stop, slab.numpy(), phases))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_step_matches_single_process(world):
    """The bench's strong-scaling step (view-sharded A, one all-gather,
    slab-sharded B) reassembles B(A(vol)) of the single process."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_step_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = load_golden("dd3d_flat")
    ref = O.dd3d("B", O.dd3d("A", g["image"], g["options"], g["angles"]), g["options"], g["angles"])
    out = np.zeros_like(ref)
    for rank, z0, z1, slab, phases in results:
        assert phases == ["projection", "gather", "backprojection"]
        out[:, :, z0:z1] = slab
    np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


@pytest.mark.gpu
def test_gpu_slab_and_view_shards_match_full_operators(cuda):
    """The CUDA operators on view shards and z-slabs reassemble the full
    projection and backprojection (single process, no collective)."""
    from xrecon_b200 import backend as BK
    g = load_golden("dd3d_flat")
    opts = torch.from_numpy(g["options"]).to(cuda)
    ang = torch.from_numpy(g["angles"]).to(cuda)
    vol = torch.from_numpy(g["image"]).to(cuda)
    full_a = BK.forward_projection3d(vol, opts, ang)
    parts = [XD.project_views(BK.forward_projection3d, vol, opts, ang, r, 3) for r in range(3)]
    assert torch.equal(torch.cat(parts, dim=2), full_a)
    full_b = BK.weighted_backward_projection3d(full_a, opts, ang)
    out = torch.empty_like(full_b)
    for r in range(3):
        zs, slab = XD.backproject_slab(BK.weighted_backward_projection3d, full_a, opts, ang, r, 3)
        out[:, :, zs] = slab
    assert float((out - full_b).norm() / full_b.norm()) < 1e-6
