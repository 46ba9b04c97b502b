"""Lane sharding over several GPUs, one process per GPU.

The reference splits a lane batch into contiguous slices per device,
weighted by capacity (src/analysis/gpu/devices.zig:181-233,
src/analysis/gpu/multi.zig:15-30), and every slice builds the same pivot tape
from the same lead lane, so results do not depend on the device count
(multi.zig:1-5). Lanes are independent: there is no collective on the data
path, only a gather of the results to rank 0 at the end.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from .decks import Netlist


def split_lanes(total: int, weights: Sequence[float]) -> List[Tuple[int, int]]:
    """Contiguous (start, count) slices of `total` lanes proportional to
    `weights`; the rounding remainder goes to the first slices."""
    w = np.asarray(weights, dtype=np.float64)
    if total <= 0 or len(w) == 0 or not np.all(w >= 0) or w.sum() <= 0:
        raise ValueError("bad split")
    raw = total * w / w.sum()
    counts = np.floor(raw).astype(int)
    rem = total - int(counts.sum())
    order = np.argsort(-(raw - counts), kind="stable")
    for i in order[:rem]:
        counts[i] += 1
    out, start = [], 0
    for c in counts:
        out.append((start, int(c)))
        start += int(c)
    return out


def shard(net: Netlist, rank: int, world: int, weights: Sequence[float] = ()) -> Tuple[Netlist, int]:
    """This rank's slice of a template's lanes, and the slice's first lane.
    Every rank keeps lane 0 of the template as its lead lane for the tape:
    the slice's netlist carries that lane first when it is not its own, and
    the caller drops it from the results (`lead_extra` = 1)."""
    slices = split_lanes(net.lanes, weights or [1.0] * world)
    start, count = slices[rank]
    idx = list(range(start, start + count))
    if start != 0:
        idx = [0] + idx
    return net.subset(idx), start


def gather_rows(local_rows: np.ndarray, start: int, lead_extra: int, group=None) -> np.ndarray:
    """All ranks' per-lane rows at rank 0, in lane order."""
    import torch.distributed as dist
    rows = local_rows[lead_extra:]
    world = dist.get_world_size(group)
    parts: List = [None] * world
    dist.all_gather_object(parts, (start, rows), group=group)
    parts.sort(key=lambda p: p[0])
    return np.concatenate([p[1] for p in parts], axis=0)
