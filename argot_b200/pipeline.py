"""Host-side driver of the device-resident path (Python over the C ABI).

``Problem`` owns the device buffers of one mesh + source set (allocated
through PyTorch, which is only the allocator and stream provider here) and
runs the hot path through libargot_b200:

    pack fields -> oct-tree (host) -> device walk: count, scan, emit rays
    -> march (columns per ray) -> per-cell rates

The rays of one target block are contiguous; ``groups`` bounds the ray
buffer by processing contiguous ranges of target blocks, the device analogue
of the reference's memory-bounded target groups
(step_radiation_tree.c:235-308).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .workload import Workload, photon_rates


def _p(t) -> int:
    return 0 if t is None else t.data_ptr()


def photon_counts(typ: int, param: float):
    lib = L.load()
    counts = np.zeros(256, np.float64)
    norm = C.c_double()
    lib.argot_b200_photon_counts(int(typ), float(param), counts.ctypes.data, C.byref(norm))
    return counts, norm.value


def tables():
    lib = L.load()
    nu = np.zeros(256, np.float64)
    cs = np.zeros((256, 3), np.float32)
    lib.argot_b200_tables(nu.ctypes.data, cs.ctypes.data)
    return nu, cs


def unit_box_grid(edge: int, lunit: float, denstonh: float) -> L.Grid:
    d = float(np.float32(1.0) / np.float32(edge))
    return L.Grid(edge, edge, edge, 0, 0, 0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0,
                  d, d, d, lunit, denstonh)


@dataclass
class RayGroup:
    b0: int
    b1: int
    base: int
    nray: int


class Problem:
    def __init__(self, wl: Workload, device: str | torch.device = "cuda:0",
                 max_group_rays: int | None = None, host_fields=None):
        """host_fields: optional pinned host tensors (dens, fHI, fHeI, fHeII)
        copied asynchronously instead of the workload's numpy arrays."""
        self.lib = L.load()
        self.wl = wl
        self.device = torch.device(device)
        self.grid = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
        self.ncell = wl.edge ** 3
        self.spectra = (np.ascontiguousarray(wl.src_spectra, np.float64) if wl.src_spectra is not None
                        else photon_rates(photon_counts, wl.src_type, wl.src_param, wl.src_rate))
        with torch.cuda.device(self.device):
            self.stream = torch.cuda.current_stream(self.device)
            if host_fields is not None:
                self.fields = [t.to(self.device, non_blocking=True) for t in host_fields]
            else:
                self.fields = [torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
                               for a in wl.fields()]
            self.packed = torch.empty(8 * self.ncell, dtype=torch.float32, device=self.device)
            self._tree = C.c_void_p()
            self._dtree = C.c_void_p()
            self._build_tree()
            self.pack()
            self._count_rays()
        self.max_group_rays = max_group_rays
        self.groups = self._make_groups(max_group_rays)

    # ------------------------------------------------------------- setup
    @property
    def sp(self):
        return C.c_void_p(self.stream.cuda_stream)

    def pack(self):
        d, a, b, c = (_p(t) for t in self.fields)
        L.check(self.lib.argot_b200_pack_fields(C.byref(self.grid), d, a, b, c, _p(self.packed),
                                                self.sp), "pack_fields")

    def _build_tree(self):
        pos = np.ascontiguousarray(self.wl.src_pos, np.float32)
        spec = np.ascontiguousarray(self.spectra, np.float64)
        L.check(self.lib.argot_b200_tree_build(C.byref(self.grid), len(pos), pos.ctypes.data,
                                               spec.ctypes.data, float(self.wl.theta),
                                               C.byref(self._tree)), "tree_build")
        L.check(self.lib.argot_b200_dev_tree_upload(self._tree, C.byref(self._dtree), self.sp),
                "dev_tree_upload")
        self.n_nodes = self.lib.argot_b200_tree_num_nodes(self._tree)
        self.n_emit = self.lib.argot_b200_tree_num_emitters(self._tree)

    def emitters(self):
        pos4 = np.zeros((self.n_emit, 4), np.float32)
        spec = np.zeros((self.n_emit, 256), np.float64)
        L.check(self.lib.argot_b200_tree_emitters(self._tree, pos4.ctypes.data, spec.ctypes.data),
                "tree_emitters")
        return pos4, spec

    def _count_rays(self):
        nb = C.c_uint64()
        L.check(self.lib.argot_b200_num_blocks(C.byref(self.grid), C.byref(nb)), "num_blocks")
        self.nblocks = nb.value
        self.blk_count = torch.zeros(self.nblocks, dtype=torch.int64, device=self.device)
        self.cell_count = torch.zeros(self.ncell, dtype=torch.int32, device=self.device)
        L.check(self.lib.argot_b200_count_rays(C.byref(self.grid), self._dtree, 0, self.nblocks,
                                               _p(self.blk_count), _p(self.cell_count), self.sp),
                "count_rays")
        self.blk_off = torch.zeros(self.nblocks + 1, dtype=torch.int64, device=self.device)
        tot = C.c_uint64()
        L.check(self.lib.argot_b200_scan_blocks(_p(self.blk_count), self.nblocks, 0,
                                                _p(self.blk_off), C.byref(tot), self.sp),
                "scan_blocks")
        self.nray = tot.value
        self.blk_off_host = self.blk_off.cpu().numpy()

    def restrict(self, b0: int, b1: int, max_rays: int | None = None):
        """Only the target blocks [b0, b1) from now on (one rank's shard)."""
        self.groups = self._make_groups(max_rays, b0, b1)
        return self.groups

    def _make_groups(self, max_rays, blk0: int = 0, blk1: int | None = None):
        off = self.blk_off_host
        blk1 = self.nblocks if blk1 is None else blk1
        if blk1 <= blk0:
            return []
        nray = int(off[blk1] - off[blk0])
        if not max_rays or nray <= max_rays:
            return [RayGroup(blk0, blk1, int(off[blk0]), nray)]
        groups, b0 = [], blk0
        while b0 < blk1:
            b1 = int(np.searchsorted(off, off[b0] + max_rays, side="right")) - 1
            b1 = max(b1, b0 + 1)
            b1 = min(b1, blk1)
            groups.append(RayGroup(b0, b1, int(off[b0]), int(off[b1] - off[b0])))
            b0 = b1
        return groups

    def alloc_group_buffers(self, group: RayGroup | None = None):
        n = max((g.nray for g in self.groups), default=0) if group is None else group.nray
        rays = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        tau = torch.empty(3 * max(n, 1), dtype=torch.float32, device=self.device)
        return rays, tau

    def emit(self, group: RayGroup, rays):
        L.check(self.lib.argot_b200_emit_rays(C.byref(self.grid), self._dtree, group.b0, group.b1,
                                              _p(self.blk_off), group.base, _p(rays), self.sp),
                "emit_rays")

    def march(self, group: RayGroup, rays, tau, precision=L.PRECISION_KAHAN, crossings=None):
        L.check(self.lib.argot_b200_march_rays(C.byref(self.grid), _p(self.packed), self._dtree,
                                               group.b0, group.b1, _p(self.blk_off), group.base,
                                               _p(rays), group.nray, _p(tau), int(precision),
                                               _p(crossings), self.sp), "march_rays")

    def rates(self, group: RayGroup, rays, tau, rates6, mode=L.RATE_EXACT_F32):
        L.check(self.lib.argot_b200_photoion_rays(C.byref(self.grid), _p(self.packed), self._dtree,
                                                  group.b0, group.b1, _p(self.blk_off), group.base,
                                                  _p(rays), group.nray, _p(tau), int(mode),
                                                  _p(rates6), self.sp), "photoion_rays")

    def set_blackbody(self):
        """Spectral temperatures of the sources (blackbodies) for the
        surrogate; other spectrum types are marked for exact integration."""
        T = np.where(self.wl.src_type == 0, self.wl.src_param, -1.0).astype(np.float32)
        L.check(self.lib.argot_b200_dev_tree_set_blackbody(self._tree, self._dtree, T.ctypes.data,
                                                           self.sp), "dev_tree_set_blackbody")

    def surrogate_work(self, nray: int | None = None):
        """Device workspace of the surrogate rates for the largest group."""
        n = max((g.nray for g in self.groups), default=0) if nray is None else nray
        nbytes = int(self.lib.argot_b200_surrogate_workspace(max(n, 1)))
        return torch.empty(nbytes // 4, dtype=torch.float32, device=self.device)

    def rates_surrogate(self, group: RayGroup, rays, tau, rates6, surrogate, counters=None, work=None):
        if work is None:
            if getattr(self, "_sur_work", None) is None or self._sur_work.numel() < 7 * group.nray:
                self._sur_work = self.surrogate_work()
            work = self._sur_work
        L.check(self.lib.argot_b200_photoion_rays_surrogate(
            C.byref(self.grid), _p(self.packed), self._dtree, surrogate.handle, group.b0, group.b1,
            _p(self.blk_off), group.base, _p(rays), group.nray, _p(tau), _p(work), _p(rates6),
            _p(counters), self.sp), "photoion_rays_surrogate")

    def smooth(self, rates6, out=None, isolated: bool = True):
        """The 27-point smoothing of smooth_photoion_rate.c on the device;
        returns `out` (a new tensor unless given)."""
        out = torch.empty_like(rates6) if out is None else out
        L.check(self.lib.argot_b200_smooth_rates(C.byref(self.grid), _p(rates6), _p(out), int(isolated),
                                                 self.sp), "smooth_rates")
        return out

    def check_device_error(self):
        L.check(self.lib.argot_b200_check_device_error(self.sp), "device error flag")

    # ------------------------------------------------------------- whole pass
    def run(self, precision=L.PRECISION_KAHAN, mode=L.RATE_EXACT_F32, rates6=None,
            buffers=None, crossings=None, keep_rays=False, overlap: int = 0):
        """march + rates over every group; returns rates6 (6, ncell).

        overlap = P > 1 (one group whose buffers hold all rays): the group
        is cut into P parts along its blocks; the march of part p+1 runs on
        one stream while the rates of part p run on another, so the
        latency-bound march and the MUFU-bound rate kernel share the GPU at
        each hand-over.  Same arithmetic: the result equals overlap = 0 bit
        for bit.  The caller's current stream is ordered after all of it."""
        if rates6 is None:
            rates6 = torch.zeros(6 * self.ncell, dtype=torch.float32, device=self.device)
        rays, tau = buffers if buffers is not None else self.alloc_group_buffers()
        if overlap > 1 and len(self.groups) == 1 and self.groups[0].nray > 0:
            return self._run_overlapped(precision, mode, rates6, rays, tau, crossings, keep_rays, overlap)
        for g in self.groups:
            if len(self.groups) > 1 or not keep_rays:
                self.emit(g, rays)
            self.march(g, rays, tau, precision, crossings)
            self.rates(g, rays, tau, rates6, mode)
        return rates6

    def part_count(self, n: int) -> int:
        """the number of parts argot_b200_run_group cuts the single group
        into for n (its block ranges of about equal ray counts)"""
        g = self.groups[0]
        off = np.asarray(self.blk_off_host, dtype=np.int64)
        cuts = [g.b0]
        for p in range(1, n):
            want = off[g.b0] + int(float(off[g.b1] - off[g.b0]) * p / n)
            b = int(np.searchsorted(off[cuts[-1]:g.b1], want, side="left")) + cuts[-1]
            if cuts[-1] < b < g.b1:
                cuts.append(b)
        return len(cuts)

    def parts(self, rays, tau, n: int):
        """The single group cut into about n parts along its blocks, each with
        its views of the ray buffer (offset base) and of the column buffer
        (three planes of the part's rays at 3 * base)."""
        g0 = self.groups[0]
        sub = self._make_groups(max(1, -(-g0.nray // n)), g0.b0, g0.b1)
        out = []
        for g in sub:
            lo = g.base - g0.base
            out.append((RayGroup(g.b0, g.b1, g.base, g.nray), rays[lo:lo + max(g.nray, 1)],
                        tau[3 * lo:3 * (lo + max(g.nray, 1))]))
        return out

    def _run_overlapped(self, precision, mode, rates6, rays, tau, crossings, keep_rays, n):
        """one call of argot_b200_run_group over the single group"""
        g = self.groups[0]
        if getattr(self, "_blk_off_host_u64", None) is None:
            self._blk_off_host_u64 = np.ascontiguousarray(self.blk_off_host, dtype=np.uint64)
        L.check(self.lib.argot_b200_run_group(
            C.byref(self.grid), _p(self.packed), self._dtree, g.b0, g.b1, _p(self.blk_off),
            self._blk_off_host_u64.ctypes.data, g.base, _p(rays), _p(tau), 0 if keep_rays else 1, precision, mode,
            n, _p(rates6), _p(crossings), self.sp), "run_group")
        return rates6

    def close(self):
        if self._dtree:
            self.lib.argot_b200_dev_tree_free(self._dtree)
            self._dtree = C.c_void_p()
        if self._tree:
            self.lib.argot_b200_tree_free(self._tree)
            self._tree = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- helpers
    def ray_table(self, rays: torch.Tensor, group: RayGroup):
        """Host view of a group's rays: (emitter, target cell (ix,iy,iz), block)."""
        w = rays[:group.nray].cpu().numpy().view(np.uint32)
        emit = (w >> 5).astype(np.int64)
        lane = (w & 31).astype(np.int64)
        off = self.blk_off_host
        blk = np.repeat(np.arange(group.b0, group.b1), np.diff(off[group.b0:group.b1 + 1]))
        e = self.wl.edge
        nbz = (e + 3) // 4
        nby = (e + 3) // 4
        bx = blk // (nby * nbz)
        by = (blk - bx * nby * nbz) // nbz
        bz = blk - bx * nby * nbz - by * nbz
        ix = bx * 2 + (lane >> 4)
        iy = by * 4 + ((lane >> 2) & 3)
        iz = bz * 4 + (lane & 3)
        return emit, np.stack([ix, iy, iz], 1).astype(np.int32), blk
