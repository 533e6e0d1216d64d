"""Multi-GPU host logic (gravlume_b200/shard.py) with two gloo ranks on the CPU: the camera and row
partitions cover a job exactly once and balance its rays, and the end-of-job collectives (max of
device times, sum of scene gradients, gather of row bands) give the single-process answers."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gravlume_b200.shard import gather_rows, max_over_ranks, shard_cameras, shard_rows, sum_scene_gradients


def test_partitions_cover_every_camera_and_row_once():
    counts = [128 * 128, 1024 * 1024, 256 * 256, 2048 * 1024, 64 * 64, 512 * 512]
    for world in (1, 2, 3, 4, 8):
        got = [list(shard_cameras(counts, world, r)) for r in range(world)]
        flat = [i for g in got for i in g]
        assert flat == list(range(len(counts)))
        for height in (1, 7, 1080, 2160):
            rows = [shard_rows(height, world, r) for r in range(world)]
            assert [i for r in rows for i in r] == list(range(height))
            assert max(len(r) for r in rows) - min(len(r) for r in rows) <= 1
    # balance: no rank holds more than the average plus the largest camera
    world = 4
    per = [sum(counts[i] for i in shard_cameras(counts, world, r)) for r in range(world)]
    assert max(per) <= sum(counts) / world + max(counts)


def test_frame_regions_cover_every_pixel_row_once():
    from gravlume_b200.shard import region_pixel_rows, shard_region

    for width, height in ((3840, 2160), (1001, 17), (8, 8), (64, 9)):
        for world in (1, 2, 3, 4, 8):
            regions = [shard_region(width, height, world, r) for r in range(world)]
            rows = [i for r in regions for i in region_pixel_rows(r, width, height)]
            assert rows == list(range(height))
            for r in regions:
                if r is not None:
                    assert r.origin[0] == 0 and r.workgroups[0] == -(-width // 8)


def _worker(rank, world, port, height, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = max_over_ranks(10.0 + rank)
        g = sum_scene_gradients(torch.tensor([1.0, 2.0, 3.0, 4.0], dtype=torch.float64) * (rank + 1))
        rows = shard_rows(height, world, rank)
        local = torch.arange(rows.start, rows.stop, dtype=torch.float64)[:, None] * torch.ones(1, 3,
                                                                                                  dtype=torch.float64)
        full = gather_rows(local, height)
        q.put((rank, t, g.tolist(), full[:, 0].tolist()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_and_gather():
    world, height = 2, 1081
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, height, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, t, g, full in out:
        assert t == 11.0
        assert g == [3.0, 6.0, 9.0, 12.0]
        assert full == [float(i) for i in range(height)]

