"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

`bench.py --gpus N` runs N independent replicas (the decode path has no exchange step); the only
collectives are the barrier around the timed region and the max-over-ranks reduction of the device
timings, and the reference arm runs on rank 0 alone.  Both are checked here without a GPU.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        got = bench.max_over_ranks(10.0 * rank + 1.5, dist, "cpu")
        # the reference arm: ranks other than 0 return at once, without work or output
        ref = bench.run_reference(None, rank, world) if rank != 0 else 0
        dist.barrier()
        out.put((rank, got, ref))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference_arm():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, ref in res:
        assert got == pytest.approx(10.0 * (world - 1) + 1.5)
        assert ref == 0


def test_max_over_ranks_without_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25
    assert os.path.exists(os.path.join(ROOT, "bench.py"))


def test_roofline_traffic_only_for_the_captured_launch_shape():
    """`roofline.traffic` comes from the committed ncu summary of the decode kernel; it is reported
    only for launches of the frame count that summary was captured on."""
    sys.path.insert(0, ROOT)
    import bench
    frames = None
    for line in open(os.path.join(ROOT, "profiles", "decode_leaf_cfg2.md")):
        if line.startswith("traffic_frames_per_launch:"):
            frames = int(line.split(":")[1])
    assert frames is not None
    assert bench.ncu_traffic(frames) > 0
    assert bench.ncu_traffic(frames + 1) is None
