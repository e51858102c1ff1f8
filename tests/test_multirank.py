"""The multi-rank host logic on CPU: world size 2 over gloo.

bench.py's multi-GPU step renders one frame per rank and gathers the
G-buffers on every rank (mb3d-rs_b200/cards.py); the step time is the
slowest rank's.  An animation is split by frames, one picture by bands of
rows, with one all_gather.  Here two CPU ranks run the same host code with
the oracle standing in for the card: the shares cover every frame and row
exactly once, and the gathered G-buffers equal the one-rank render.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "mb3d-rs_b200")]
import cards  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("n", [0, 1, 7, 240, 1080])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shares_cover_every_item_once(n, world):
    seen = []
    for r in range(world):
        a, b = cards.share(n, r, world)
        assert 0 <= a <= b <= n
        seen.extend(range(a, b))
        sizes = [cards.share(n, k, world)[1] - cards.share(n, k, world)[0] for k in range(world)]
        assert max(sizes) - min(sizes) <= 1
    assert seen == list(range(n))
    with pytest.raises(ValueError):
        cards.share(n, world, world)


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path[:0] = [ROOT, os.path.join(ROOT, "mb3d-rs_b200"), os.path.join(ROOT, "oracle")]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    import cards
    import mb3dcu
    import oracle_py as O
    import scenes
    rec = mb3dcu.SILIGHT.itemsize
    # an animation split by frames (the oracle renders this rank's frames)
    frames = [scenes.scaled(f, 40, 24) for f in scenes.c4_frames(5)]
    f0, f1 = cards.share(len(frames), rank, world)
    local = np.concatenate([O.march(f, mb3dcu.SILIGHT) for f in frames[f0:f1]])
    counts = [(cards.share(5, r, world)[1] - cards.share(5, r, world)[0]) * 40 * 24 for r in range(world)]
    allf = cards.gather(local, counts, rec).numpy().tobytes()
    # one picture split by bands of rows
    sc = scenes.scaled(scenes.c2_hybrid(), 48, 27)
    row0, rows = cards.row_band(sc.height, rank, world)
    band = O.march(sc, mb3dcu.SILIGHT, row0, rows)
    counts = [cards.row_band(27, r, world)[1] * 48 for r in range(world)]
    allr = cards.gather(band, counts, rec).numpy().tobytes()
    # bench.py's step: one frame per rank, the slowest rank's time
    scb = bench.frame(rank, 0.1)
    worst = bench.max_over_ranks(10.0 + rank * 5.0, world, "cpu")
    q.put((rank, allf, allr, tuple(scb.vgrads[2]), worst))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_split_and_gather():
    import mb3dcu
    import oracle_py as O
    import scenes
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (_, f_a, r_a, v0, m0), (_, f_b, r_b, v1, m1) = res
    frames = [scenes.scaled(f, 40, 24) for f in scenes.c4_frames(5)]
    want_f = np.concatenate([O.march(f, mb3dcu.SILIGHT) for f in frames]).tobytes()
    want_r = O.march(scenes.scaled(scenes.c2_hybrid(), 48, 27), mb3dcu.SILIGHT).tobytes()
    assert f_a == f_b == want_f
    assert r_a == r_b == want_r
    assert v0 != v1  # each rank's own camera
    assert m0 == m1 == 15.0
