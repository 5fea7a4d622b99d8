"""The sharded device path (argot_b200/shard.py with argot_b200.pipeline).

Every light ray ends in one target cell, so a rank that computes only the
target blocks of its x-slab range produces exactly the rates the whole-mesh
run gives those cells.  Checked two ways on the one GPU a test gets:

* one process computes each range of shard.partition in turn
  (Problem.restrict) and the slabs, put together, equal the whole-mesh run
  bit for bit, for the compensated FP32 path and the reference-order FP64
  path;
* two gloo ranks each drive the device path for their own range, exchange
  their slabs through shard.gather_rates (host copies) and take the
  convergence verdict through shard.converged; both end with the whole-mesh
  field.  The ranks' kernels never wait on one another (the exchange is on
  the host after each rank's pass), so sharing one GPU is safe.
"""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WS = 2


def _problem_rates(wl, precision, mode, part=None):
    import torch
    from argot_b200.pipeline import Problem
    pb = Problem(wl)
    if part is not None:
        pb.restrict(*part)
    rays, tau = pb.alloc_group_buffers()
    rates = torch.zeros(6 * pb.ncell, dtype=torch.float32, device="cuda")
    for g in pb.groups:
        pb.emit(g, rays)
        pb.march(g, rays, tau, precision)
        pb.rates(g, rays, tau, rates, mode)
    torch.cuda.synchronize()
    pb.check_device_error()
    counts = pb.blk_count.cpu().numpy()
    pb.close()
    return rates.view(6, -1).cpu().numpy(), counts


@pytest.mark.parametrize("ws", [2, 3, 5])
def test_slabs_put_together_equal_the_whole_run(cuda_ok, ws):
    from argot_b200 import _lib as L
    from argot_b200 import shard
    from argot_b200 import workload as W
    wl = W.tiny(32, 20, seed=23, sigma_ln=1.2)
    for prec, mode in ((L.PRECISION_KAHAN, L.RATE_EXACT_F32), (L.PRECISION_REFERENCE, L.RATE_EXACT_F64)):
        whole, counts = _problem_rates(wl, prec, mode)
        parts = shard.partition(counts, ws, wl.edge)
        got = np.full_like(whole, np.nan)
        for b0, b1 in parts:
            c0, c1 = shard.cells_of(b0, b1, wl.edge)
            if c1 > c0:
                slab, _ = _problem_rates(wl, prec, mode, (b0, b1))
                got[:, c0:c1] = slab[:, c0:c1]
        assert np.array_equal(got, whole), (ws, prec, mode)


# ------------------------------------------------------------ two gloo ranks
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_pass(rank, ws, out_dir):
    import torch
    from argot_b200 import _lib as L
    from argot_b200 import shard
    from argot_b200 import workload as W
    torch.cuda.set_device(0)
    wl = W.tiny(32, 16, seed=29, sigma_ln=1.0)
    _, counts = _problem_rates(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32, (0, 0))
    parts = shard.partition(counts, ws, wl.edge)
    ranges = [shard.cells_of(b0, b1, wl.edge) for b0, b1 in parts]
    mine, _ = _problem_rates(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32, parts[rank])
    full = shard.gather_rates(torch.from_numpy(np.ascontiguousarray(mine).ravel()), ranges).numpy()
    np.save(os.path.join(out_dir, f"rates_{rank}.npy"), full)
    # a second pass after a change of the field: every rank sees the same
    # verdict from its own cells' change
    wl.fHI = (wl.fHI * np.float32(0.9)).astype(np.float32)
    mine2, _ = _problem_rates(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32, parts[rank])
    c0, c1 = ranges[rank]
    ch = shard.rate_change(torch.from_numpy(mine[:, c0:c1].copy()), torch.from_numpy(mine2[:, c0:c1].copy()),
                           floor=1e-30)
    verdicts = (shard.converged(ch, 1e-12), shard.converged(ch, 10.0))
    np.save(os.path.join(out_dir, f"change_{rank}.npy"), np.array([ch]))
    return all(c1 > c0 for c0, c1 in ranges) and verdicts == (False, True)


def _worker(rank, ws, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=120))
    try:
        ok = _rank_pass(rank, ws, out_dir)
        with open(os.path.join(out_dir, f"ok_{rank}"), "w") as f:
            f.write("1" if ok else "0")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_drive_the_device_path(cuda_ok):
    import torch.multiprocessing as mp
    from argot_b200 import _lib as L
    from argot_b200 import workload as W
    wl = W.tiny(32, 16, seed=29, sigma_ln=1.0)
    whole, _ = _problem_rates(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(WS, _free_port(), d), nprocs=WS, join=True, start_method="spawn")
        flags = [open(os.path.join(d, f"ok_{r}")).read() for r in range(WS)]
        got = [np.load(os.path.join(d, f"rates_{r}.npy")) for r in range(WS)]
        changes = [float(np.load(os.path.join(d, f"change_{r}.npy"))[0]) for r in range(WS)]
    assert flags == ["1"] * WS
    for g in got:
        assert np.array_equal(g, whole)
    assert all(c > 0 for c in changes)
