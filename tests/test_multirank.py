"""The multi-rank host logic of bench.py on CPU: world size 2 over gloo.

With N GPUs every rank renders its own frame (its own camera seed) and the
step time is the slowest rank's; these are the only cross-rank steps (no
collective touches the pictures).  Here two CPU ranks check that they pick
different frames of the same size and that the max over ranks is taken.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    import datetime
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "mb3d-rs_b200")]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    sc = bench.frame(rank, 0.1)
    ms = 10.0 + rank * 5.0
    worst = bench.max_over_ranks(ms, world, "cpu")
    q.put((rank, sc.width, sc.height, tuple(sc.vgrads[2]), worst))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_pick_their_frames_and_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    (r0, w0, h0, v0, m0), (r1, w1, h1, v1, m1) = res
    assert (w0, h0) == (w1, h1)
    assert v0 != v1  # each rank's own camera
    assert m0 == m1 == 15.0
