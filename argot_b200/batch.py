"""Many independent problems (meshes + source sets of uneven size) in one
persistent launch (argot_b200_batch_*, csrc/batch.cu).

Each problem is prepared by the single-problem driver (``Problem``: packed
fields, tree, ray counts and offsets, and every ray emitted once, since the
rays depend only on the tree and the mesh geometry); a step is then one
launch that marches and integrates every ray of every problem, directly or
as a replayed CUDA graph.  The tile length, warps per CTA and CTAs per SM
come from the library's autotuner, which times candidates on the batch.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .pipeline import Problem, _p


class Batch:
    def __init__(self, workloads, device="cuda:0"):
        self.lib = L.load()
        self.device = torch.device(device)
        self.problems = []
        self.rays = []
        self.rates = []
        for wl in workloads:
            pb = Problem(wl, self.device)
            rays = torch.empty(max(pb.nray, 1), dtype=torch.int32, device=self.device)
            pb.emit(pb.groups[0], rays)
            self.problems.append(pb)
            self.rays.append(rays)
            self.rates.append(torch.zeros(6 * pb.ncell, dtype=torch.float32, device=self.device))
        self._offs = [pb.blk_off_host.astype("uint64") for pb in self.problems]
        arr = (L.BatchProblem * len(self.problems))()
        for i, pb in enumerate(self.problems):
            arr[i] = L.BatchProblem(pb.grid, _p(pb.packed), pb._dtree.value, _p(pb.blk_off),
                                    self._offs[i].ctypes.data, _p(self.rays[i]), _p(self.rates[i]))
        self.handle = C.c_void_p()
        L.check(self.lib.argot_b200_batch_create(arr, len(arr), C.byref(self.handle)), "batch_create")

    @property
    def sp(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def nray(self):
        return sum(pb.nray for pb in self.problems)

    @property
    def ncell(self):
        return sum(pb.ncell for pb in self.problems)

    def config(self):
        c = L.BatchConfig()
        L.check(self.lib.argot_b200_batch_get_config(self.handle, C.byref(c)), "batch_get_config")
        return c.as_dict()

    def configure(self, warps_per_cta=8, ctas_per_sm=0, blocks_per_item=4, order=0, mode=0, parts=8):
        """mode 0: fused march + rates in one persistent kernel; 1: split into
        a persistent march kernel and a persistent rate kernel overlapped
        over `parts` parts of the tile list."""
        c = L.BatchConfig(warps_per_cta, ctas_per_sm, blocks_per_item, order, mode, parts)
        L.check(self.lib.argot_b200_batch_configure(self.handle, C.byref(c)), "batch_configure")

    def tune(self, reps: int = 1):
        c = L.BatchConfig()
        ms = C.c_float()
        L.check(self.lib.argot_b200_batch_tune(self.handle, reps, C.byref(c), C.byref(ms), self.sp),
                "batch_tune")
        return c.as_dict(), ms.value

    def run(self, crossings=None):
        L.check(self.lib.argot_b200_batch_run(self.handle, _p(crossings), self.sp), "batch_run")

    def graph_launch(self):
        L.check(self.lib.argot_b200_batch_graph_launch(self.handle, self.sp), "batch_graph_launch")

    def check_device_error(self):
        L.check(self.lib.argot_b200_check_device_error(self.sp), "device error flag")

    def close(self):
        if self.handle:
            self.lib.argot_b200_batch_free(self.handle)
            self.handle = C.c_void_p()
        for pb in self.problems:
            pb.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
