"""One render split across ranks by slabs of the screen.

The screen's pixels are numbered with the first axis fastest, so the rows of
the last axis are contiguous runs of pixels and a slab of rows [begin, end)
is the pixel range [begin * row, end * row).  Rank r of W renders the slab
slab_rows(rows, r, W): the paths of its rows and of one row either side
(the pixel filter reaches one pixel, and every path's stream is fixed by
(seed, pass, pixel, sample), so those halo paths are recomputed, not
exchanged), and the estimator of its own rows.  The slabs' images put
together in rank order (assemble) are the whole-screen image bit for bit.
Nothing is exchanged while rendering; one gather of the slab images ends
the render.
"""

from __future__ import annotations

import numpy as np


def slab_rows(rows: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [begin, end) of the last screen axis for `rank` of `world`: as
    equal as the rows allow, the first `rows % world` ranks one row more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    if rows < world:
        raise ValueError(f"{rows} rows cannot be split across {world} ranks")
    base, extra = divmod(rows, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def source_rows(rows: int, begin: int, end: int) -> tuple[int, int]:
    """The rows whose paths a slab renders: its own and one on either side."""
    return max(0, begin - 1), min(rows, end + 1)


def pixel_range(size, begin: int, end: int) -> tuple[int, int]:
    """Pixel index range of rows [begin, end) of a screen of `size`."""
    row = int(np.prod(size[:-1]))
    return begin * row, end * row


def assemble(tiles: list[np.ndarray]) -> np.ndarray:
    """The slabs' images (pixels x channels), in rank order, as one image."""
    return np.concatenate(tiles, axis=0)


def gather_image(tile: np.ndarray, rank: int, world: int, rows: int, size) -> np.ndarray | None:
    """Gathers every rank's slab image to rank 0 (torch.distributed, whatever
    the process group's backend) and returns the whole image there, None on
    the other ranks.  Slabs differ in length by at most a row, so each is
    padded to the longest before the gather."""
    import torch
    import torch.distributed as dist

    row = int(np.prod(size[:-1]))
    longest = (rows // world + (1 if rows % world else 0)) * row
    padded = np.zeros((longest, tile.shape[1]), tile.dtype)
    padded[: len(tile)] = tile
    t = torch.from_numpy(padded)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    parts = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, parts, dst=0)
    if rank != 0:
        return None
    tiles = []
    for r in range(world):
        b, e = slab_rows(rows, r, world)
        tiles.append(parts[r].cpu().numpy()[: (e - b) * row])
    return assemble(tiles)
