"""A render spread over several GPUs (one process per GPU), with one gather.

mb3d-rs spreads one picture over its graphics cards by work stealing: every
card takes the next band of rows from a shared board until the picture is
done (render.rs:1390-1470 `Board::steal`, gpu.rs:2775 `on_cards`), and an
animation is a list of frames rendered one after the other
(frames.rs:467 `render_frames`).  Pixels and frames are independent, so
on B200s the split is fixed up front and the only cross-GPU step is the
gather of the results:

  - frames: rank r renders frames [f0, f1) of the animation (contiguous
    shares that differ by at most one frame) through one
    mb3d_cu_render_frames call, and the G-buffers are gathered;
  - rows: rank r marches the band of rows [row0, row0 + rows) of one
    picture, and the bands are gathered in row order.

The gather is one torch.distributed all_gather of equal-sized byte buffers
(the shares are padded to the largest one), over NCCL for device buffers
(NVLink) or gloo for host buffers; there is no other collective on the
data path and no TMA multicast anywhere.
"""
import numpy as np


def share(n, rank, world):
    """The contiguous share [start, stop) of n items for `rank` of `world`
    ranks: the first n % world ranks take one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def row_band(height, rank, world):
    """(row0, rows) of this rank's band of a picture `height` rows high."""
    a, b = share(height, rank, world)
    return a, b - a


def gather(local, counts, item_bytes, device=None):
    """All ranks' shares in rank order: `local` is this rank's share (a
    numpy array or torch tensor of counts[rank] items of item_bytes bytes);
    returns a torch uint8 tensor of sum(counts) items on every rank (on
    `device`, or where `local` is)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    rank = dist.get_rank()
    if len(counts) != world:
        raise ValueError("one count per rank")
    if isinstance(local, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(local).view(np.uint8).reshape(-1))
    else:
        t = local.reshape(-1).view(torch.uint8)
    if device is not None:
        t = t.to(device)
    if t.numel() != counts[rank] * item_bytes:
        raise ValueError("the local share's size is not counts[rank] items")
    most = max(counts) * item_bytes
    pad = torch.zeros(most, dtype=torch.uint8, device=t.device)
    pad[: t.numel()] = t
    parts = [torch.empty(most, dtype=torch.uint8, device=t.device) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([parts[r][: counts[r] * item_bytes] for r in range(world)])


def render_frames_share(card, frames, rank, world, precision, tune=None, out=None):
    """This rank's frames of the animation, rendered in one call: returns
    (start, stop, G-buffer of those frames)."""
    f0, f1 = share(len(frames), rank, world)
    if f1 == f0:
        return f0, f1, None
    return f0, f1, card.render_frames(frames[f0:f1], precision, tune, out=out)


def march_band(card, scene, rank, world, precision, out=None):
    """This rank's band of rows of the picture: (row0, rows, G-buffer band)."""
    row0, rows = row_band(scene.height, rank, world)
    if rows == 0:
        return row0, rows, None
    return row0, rows, card.march(scene, precision, row0=row0, rows=rows, out=out)
