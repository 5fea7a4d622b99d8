"""Multi-rank host logic on CPU with gloo (world size 2): the shard
partition of target blocks, the all-gather of rate slabs, the field
broadcast, bench.py's max/sum over ranks, and the property the sharding
rests on -- the rays of disjoint target ranges are independent -- checked
with the reference's own C (single-threaded, so its per-cell sums are
ordered) on a 16^3 mesh: each rank runs its own cell range, the gathered
rates equal one run over the whole mesh bit for bit."""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest

from argot_b200 import shard

WS = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


# ------------------------------------------------------------ partition
@pytest.mark.parametrize("edge,ws", [(16, 1), (16, 2), (16, 3), (17, 4), (10, 8), (4, 5)])
def test_partition_covers_blocks_once(edge, ws):
    S, ns = shard.blocks_per_slab(edge), shard.num_slabs(edge)
    rng = np.random.default_rng(edge * 31 + ws)
    counts = rng.integers(0, 500, S * ns)
    parts = shard.partition(counts, ws, edge)
    assert len(parts) == ws
    assert parts[0][0] == 0 and parts[-1][1] == S * ns
    for (a0, a1), (b0, b1) in zip(parts, parts[1:]):
        assert a1 == b0
    for b0, b1 in parts:
        assert b0 <= b1 and b0 % S == 0
        c0, c1 = shard.cells_of(b0, b1, edge)
        assert 0 <= c0 <= c1 <= edge ** 3
    cells = [shard.cells_of(b0, b1, edge) for b0, b1 in parts]
    assert cells[0][0] == 0 and cells[-1][1] == edge ** 3
    assert all(x[1] == y[0] for x, y in zip(cells, cells[1:]))


def test_partition_balance():
    edge, ws = 64, 4
    S, ns = shard.blocks_per_slab(edge), shard.num_slabs(edge)
    rng = np.random.default_rng(0)
    counts = rng.integers(50, 150, S * ns).astype(np.float64)
    counts[: 4 * S] *= 20  # a dense corner
    parts = shard.partition(counts, ws, edge)
    w = np.array([counts[b0:b1].sum() for b0, b1 in parts])
    slab = counts.reshape(ns, S).sum(1).max()
    # every cut lands within one slab of the balanced position
    assert np.all(np.abs(w - counts.sum() / ws) <= slab * 1.0001)


def test_partition_rejects_bad_input():
    with pytest.raises(ValueError):
        shard.partition(np.ones(10), 2, 16)
    with pytest.raises(ValueError):
        shard.cells_of(1, 64, 16)


def test_cells_of_matches_block_order():
    """Cells of a slab range are exactly the target cells of its blocks
    (block = bx * nby * nbz + by * nbz + bz, lane = lz + 4 ly + 16 lx)."""
    edge = 10
    S = shard.blocks_per_slab(edge)
    nb = (edge + 3) // 4
    b0, b1 = S, 3 * S
    cells = set()
    for b in range(b0, b1):
        bx, r = divmod(b, nb * nb)
        by, bz = divmod(r, nb)
        for lane in range(32):
            ix, iy, iz = 2 * bx + (lane >> 4), 4 * by + ((lane >> 2) & 3), 4 * bz + (lane & 3)
            if ix < edge and iy < edge and iz < edge:
                cells.add(iz + edge * (iy + edge * ix))
    c0, c1 = shard.cells_of(b0, b1, edge)
    assert cells == set(range(c0, c1))


# ------------------------------------------------------------ gloo ranks
def _task_gather(rank, ws, arg):
    import torch
    edge = 10
    S, ns = shard.blocks_per_slab(edge), shard.num_slabs(edge)
    counts = np.random.default_rng(1).integers(0, 100, S * ns)
    parts = shard.partition(counts, ws, edge)
    ranges = [shard.cells_of(b0, b1, edge) for b0, b1 in parts]
    ncell = edge ** 3
    full = (np.arange(6)[:, None] * 1e4 + np.arange(ncell)[None, :]).astype(np.float32)
    mine = np.full((6, ncell), -1.0, np.float32)  # other ranks' cells hold garbage
    c0, c1 = ranges[rank]
    mine[:, c0:c1] = full[:, c0:c1]
    out = shard.gather_rates(torch.from_numpy(mine.ravel()), ranges)
    return np.array_equal(out.numpy(), full)


def _task_broadcast(rank, ws, arg):
    import torch
    x = torch.arange(64, dtype=torch.float32) if rank == 0 else torch.zeros(64)
    shard.broadcast_field(x, 0)
    return bool(torch.equal(x, torch.arange(64, dtype=torch.float32)))


def _task_reductions(rank, ws, arg):
    import bench
    bench.barrier(ws)
    mx = bench.allmax(ws, 1.5 + rank)
    sm = bench.allsum(ws, 1.5 + rank)
    return mx == 1.5 + ws - 1 and sm == sum(1.5 + r for r in range(ws))


def _task_sharded_reference(rank, ws, out_dir):
    import torch
    from argot_b200 import workload as W
    from oracle.oracle import RefLib
    wl = W.tiny(16, 6, seed=7)
    R = RefLib(16)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    edge = wl.edge
    S, ns = shard.blocks_per_slab(edge), shard.num_slabs(edge)
    # balance by the reference's own ray counts per cell, summed per block slab
    _, per_cell = R.count_rays(0, edge ** 3, per_cell=True)
    per_slab = per_cell.astype(np.float64).reshape(ns, -1).sum(1)
    counts = np.repeat(per_slab / S, S)
    parts = shard.partition(counts, ws, edge)
    ranges = [shard.cells_of(b0, b1, edge) for b0, b1 in parts]
    c0, c1 = ranges[rank]
    R.zero_rates()
    if c1 > c0:
        R.run_range(c0, c1, True, want=())
    mine = R.get_rates()
    out = shard.gather_rates(torch.from_numpy(mine.ravel()), ranges).numpy()
    np.save(os.path.join(out_dir, f"sharded_{rank}.npy"), out)
    return all(c1 > c0 for c0, c1 in ranges)


def _task_converged(rank, ws, arg):
    """every rank reaches the same verdict from its own cells' change"""
    import torch
    prev = torch.ones(6 * 100)
    cur = prev.clone()
    cur[rank] = 1.0 + 1e-3 * (rank + 1)   # rank r changed by (r + 1) 1e-3
    ch = shard.rate_change(prev, cur)
    loose = shard.converged(ch, 5e-3)      # max change 2e-3 <= 5e-3
    tight = shard.converged(ch, 1.5e-3)    # rank 1's 2e-3 > 1.5e-3 for everyone
    c = float(cur[rank])
    return loose and not tight and abs(ch - (c - 1.0) / c) < 1e-7


TASKS = {"gather": _task_gather, "broadcast": _task_broadcast, "reductions": _task_reductions,
         "converged": _task_converged, "sharded_reference": _task_sharded_reference}


def _worker(rank, ws, port, task, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        ok = TASKS[task](rank, ws, out_dir)
        with open(os.path.join(out_dir, f"{task}_{rank}.ok"), "w") as f:
            f.write("1" if ok else "0")
    finally:
        dist.destroy_process_group()


def _run(task):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(WS, _free_port(), task, d), nprocs=WS, join=True,
                           start_method="spawn")
        flags = [open(os.path.join(d, f"{task}_{r}.ok")).read() for r in range(WS)]
        arrays = [np.load(os.path.join(d, f"sharded_{r}.npy")) for r in range(WS)
                  if os.path.exists(os.path.join(d, f"sharded_{r}.npy"))]
    return flags, arrays


@pytest.mark.parametrize("task", ["gather", "broadcast", "reductions", "converged"])
def test_gloo_exchange(task):
    flags, _ = _run(task)
    assert flags == ["1"] * WS


def test_sharded_reference_equals_whole_mesh_run():
    from conftest import ref_lib
    from argot_b200 import workload as W
    R = ref_lib(16)
    wl = W.tiny(16, 6, seed=7)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    R.zero_rates()
    R.run_range(0, wl.edge ** 3, True, want=())
    whole = R.get_rates()
    assert np.all(whole[0] > 0)
    flags, arrays = _run("sharded_reference")
    assert flags == ["1"] * WS  # every rank got a non-empty shard
    for a in arrays:
        assert np.array_equal(a, whole)
