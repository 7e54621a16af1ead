"""A frame split by points over ranks (sharded.render_point_sharded), run as
gloo ranks on CPU with the oracle's HQS stages standing in for the GPU
stages: every rank's image, depth and accumulator planes equal the oracle's
single render of the whole cloud, bit for bit.  Also the bench's rank
helpers under gloo."""
import importlib
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

from scenes import blob_cloud, look_at_reverse_z

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
W, H = 96, 72


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene(orc):
    pos, rgba = blob_cloud(40000, 17)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512)
    cfg = orc.Config(depthTolerance=0.02, holeFillIterations=1,
                     backgroundColor=(0.1, 0.2, 0.3, 1.0))
    view, proj = look_at_reverse_z((1.2, 0.7, 2.0), aspect=W / H)
    files = orc.update_files(packed.files, orc.mat4_mul(proj, view),
                             np.eye(4, dtype=np.float32))
    return packed, cfg, view, proj, files


def _rank_main(rank, world, port, out_dir, holes):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist

    import oracle as orc
    sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        packed, cfg, view, proj, files = _scene(orc)
        cfg.holeFillIterations = holes
        lo, hi = sharded.shard_range(len(packed.batches), rank, world)
        batches = packed.batches.copy()
        batches["state"][:lo] = 0  # non-resident: not this rank's part
        batches["state"][hi:] = 0
        cloud = orc.Cloud(batches, files, packed.xyzLow, packed.xyzMed, packed.xyzHigh,
                          packed.colors, packed.levels)
        depth = np.zeros(W * H, np.uint32)
        accum = np.zeros(W * H * 4, np.uint32)
        rgba = np.zeros(W * H * 4, np.uint8)
        depthf = np.zeros(W * H, np.float32)

        def run_stage(stage):
            orc.hqs_stage(cloud, cfg, view, proj, W, H, stage, depth, accum, rgba, depthf)

        def flip():
            np.bitwise_xor(depth, np.uint32(0x80000000), out=depth)

        sharded.render_point_sharded(run_stage, torch.from_numpy(depth.view(np.int32)),
                                     torch.from_numpy(accum.view(np.int32)), flip)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), depth=depth, accum=accum, rgba=rgba,
                 depthf=depthf, part=np.array([lo, hi]))
    finally:
        dist.destroy_process_group()


def _run_ranks(target, world, args):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port) + args) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


@pytest.mark.parametrize("world,holes", [(2, 1), (3, 0)])
def test_point_sharded_frame_matches_single_render(orc, tmp_path, world, holes):
    _run_ranks(_rank_main, world, (str(tmp_path), holes))
    packed, cfg, view, proj, files = _scene(orc)
    cfg.holeFillIterations = holes
    full = orc.render(packed.cloud(files), cfg, view, proj, W, H)
    assert full.accum[..., 3].sum() > 1000
    parts = []
    for r in range(world):
        d = np.load(os.path.join(tmp_path, f"rank{r}.npz"))
        parts.append(tuple(d["part"]))
        assert np.array_equal(d["depth"], full.depth.reshape(-1)), r
        assert np.array_equal(d["accum"], full.accum.reshape(-1)), r
        assert np.array_equal(d["rgba"], full.rgba.reshape(-1)), r
        assert np.array_equal(d["depthf"].view(np.uint32), full.depthf.reshape(-1).view(np.uint32))
    # The parts tile the batch list.
    assert parts[0][0] == 0 and parts[-1][1] == len(packed.batches)
    assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
    assert all(hi > lo for lo, hi in parts)


def test_shard_range_partitions():
    sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
    for n in (0, 1, 7, 9766):
        for world in (1, 2, 3, 8):
            got = [sharded.shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(got[i][1] == got[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharded.shard_range(5, 2, 2)


def _bench_rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    bench = importlib.import_module("bench")
    d = bench.Dist(backend="gloo")
    try:
        got = d.max(float(rank) + 0.5)
        d.barrier()
        order = bench.pose_order(d.rank, d.world, 3 + 5, 32)
        np.save(os.path.join(out_dir, f"b{rank}.npy"), np.array([got] + order, np.float64))
    finally:
        d.close()


def test_bench_rank_helpers_under_gloo(tmp_path):
    world = 2
    _run_ranks(_bench_rank_main, world, (str(tmp_path),))
    rows = [np.load(os.path.join(tmp_path, f"b{r}.npy")) for r in range(world)]
    assert all(r[0] == world - 0.5 for r in rows)  # max over ranks
    poses = [list(r[1:].astype(int)) for r in rows]
    # Ranks draw different poses (interleaved), each pose index in range.
    assert poses[0] != poses[1]
    assert all(0 <= p < 32 for ps in poses for p in ps)
    assert poses[0][:4] == [0, 2, 4, 6] and poses[1][:4] == [1, 3, 5, 7]
