"""One problem's target cells sharded over ranks (one process per GPU).

Every light ray ends in exactly one target cell, so the rays of disjoint
target ranges are independent: a rank marches and integrates only the rays
of its own x-slab of target blocks, with the whole field and the source
tree replicated on its GPU, and writes the rates of its own cells.  The
exchange steps of a radiation iteration around that are

* ``broadcast_field``: the packed field from the rank that holds the
  update, once per iteration (the chemistry between iterations changes the
  ionised fractions);
* ``gather_rates``: every rank's slab of the six rate planes into the whole
  field, only when the host wants the whole mesh.

The reference splits rays over MPI domains by segment and sums the columns
with one-sided RMA (src/accum_optical_depth.c:89-139), and its intra-node
multi-GPU path computes every ray's rates on every GPU
(src/calc_photoion_rate_cuda.cu:143-193); neither is needed here.

Target blocks are 2x4x4 cells, ordered x-major (block = bx * nby * nbz +
by * nbz + bz), so a range of whole x-slabs of blocks is a contiguous range
of cells in the mesh order (iz fastest, src/calc_optical_depth.c:18).
"""
from __future__ import annotations

import numpy as np


def blocks_per_slab(edge: int) -> int:
    """Blocks in one x-slab (two cells thick)."""
    return ((edge + 3) // 4) ** 2


def num_slabs(edge: int) -> int:
    return (edge + 1) // 2


def partition(counts, ws: int, edge: int):
    """Contiguous, slab-aligned block ranges [(b0, b1)] * ws balanced by
    `counts` (rays per block, or any per-block work estimate).  Ranges may
    be empty when there are more ranks than slabs."""
    counts = np.asarray(counts, np.float64)
    S = blocks_per_slab(edge)
    ns = num_slabs(edge)
    nblocks = counts.size
    if nblocks != S * ns:
        raise ValueError(f"{nblocks} block counts for a {edge}^3 mesh (want {S * ns})")
    if ws < 1:
        raise ValueError("ws must be >= 1")
    w = counts.reshape(ns, S).sum(1)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, ws):
        target = total * r / ws
        # the slab boundary nearest to the balanced cut, never going back
        s = int(np.searchsorted(cum, target))
        if s > 0 and abs(cum[s - 1] - target) <= abs(cum[min(s, ns)] - target):
            s -= 1
        cuts.append(min(max(s, cuts[-1]), ns))
    cuts.append(ns)
    return [(cuts[r] * S, cuts[r + 1] * S) for r in range(ws)]


def cells_of(b0: int, b1: int, edge: int):
    """Cell index range [c0, c1) of a slab-aligned block range."""
    S = blocks_per_slab(edge)
    if b0 % S or (b1 % S and b1 != S * num_slabs(edge)):
        raise ValueError("block range is not slab-aligned")
    ix0 = min(edge, 2 * (b0 // S))
    ix1 = min(edge, 2 * ((b1 + S - 1) // S))
    return ix0 * edge * edge, ix1 * edge * edge


def gather_rates(rates6, cell_ranges, group=None):
    """All-gather of every rank's slab of the six rate planes.

    rates6: flat tensor (6 * ncell) holding this rank's slab (other cells
    are ignored); cell_ranges: [(c0, c1)] per rank.  Returns a new (6, ncell)
    tensor with every rank's slab in place, on every rank.  Works with the
    NCCL (device tensors) and gloo (host tensors) backends."""
    import torch
    import torch.distributed as dist
    ws = dist.get_world_size(group)
    rank = dist.get_rank(group)
    planes = rates6.view(6, -1)
    ncell = planes.shape[1]
    L = max(c1 - c0 for c0, c1 in cell_ranges)
    c0, c1 = cell_ranges[rank]
    mine = torch.zeros((6, max(L, 1)), dtype=planes.dtype, device=planes.device)
    mine[:, :c1 - c0] = planes[:, c0:c1]
    bufs = [torch.empty_like(mine) for _ in range(ws)]
    dist.all_gather(bufs, mine, group=group)
    out = torch.zeros((6, ncell), dtype=planes.dtype, device=planes.device)
    for r, (a, b) in enumerate(cell_ranges):
        out[:, a:b] = bufs[r][:, :b - a]
    return out


def broadcast_field(packed, src: int = 0, group=None):
    """The packed field (argot_b200_pack_fields layout) from rank `src` to
    every rank, in place."""
    import torch.distributed as dist
    dist.broadcast(packed, src, group=group)
    return packed


def rate_change(prev6, cur6, floor: float = 0.0) -> float:
    """Largest relative change of the six rate planes between two passes of
    the iteration (|cur - prev| / |cur| over the cells whose |cur| exceeds
    `floor`), on this rank's cells."""
    import torch
    d = (cur6 - prev6).abs()
    m = cur6.abs()
    keep = m > floor
    if not bool(keep.any()):
        return 0.0
    return float(torch.max(d[keep] / m[keep]).item())


def converged(local_change: float, tol: float, group=None) -> bool:
    """The all-reduce (MAX) of the per-rank changes against tol, identical on
    every rank: the convergence test of the radiation iteration when the
    target cells are sharded over ranks."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([local_change], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return bool(t.item() <= tol)
