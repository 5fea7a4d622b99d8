"""Parity on sampled target cells of a large problem (test infrastructure).

A full run of ARGOT's own C (O1) on the largest workloads (up to 3.3e9
light rays) takes hours on the host, but the reference's own group loop
computes any range of target cells on its own: ``setup_light_ray_range``
(src/setup_light_ray_tree.c:397) builds the light rays of the cells
[im_start, im_end), which then go through calc_optical_depth,
accum_optical_depth and calc_photoion_rate (src/calc_ARGOT_part as the
reference's step_radiation_tree.c:286-300 runs it).  Every ray ends in one
target cell, so the per-cell rates of a range are complete.

``SampledParity`` runs O1 on seeded runs of consecutive target cells along
z (contiguous in the reference's cell order and in this library's target
blocks), the FP64 precision oracle (``orc_march_f64`` + ``orc_photoion_f64``)
on O1's rays of those cells, and the device path (``argot_b200.pipeline``)
on the target blocks that contain them, and compares on the sampled cells:

* the per-cell ray lists (the reference's emitters in its order),
* the reference-order columns, bit for bit,
* the FP64 rates against O1's rates,
* the compensated (Kahan) columns against the FP64 march,
* the FP32 and surrogate rates against the FP64 oracle pipeline.

Only tests/, ``__graft_entry__.smoke`` and bench.py's checks import this
module; the product never does.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle, RefLib, unit_box_grid

NAMES = ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII")


def z_runs(edge: int, nruns: int, length: int, seed: int):
    """Seeded runs of `length` consecutive target cells along z:
    (ix, iy, iz0, iz1)."""
    rng = np.random.default_rng(seed)
    length = min(length, edge)
    runs = []
    for _ in range(nruns):
        ix, iy = (int(v) for v in rng.integers(0, edge, 2))
        iz0 = int(rng.integers(0, edge - length + 1))
        runs.append((ix, iy, iz0, iz0 + length))
    return runs


def rel_err(got, want, floor=0.0):
    """Largest |got - want| / |want| over the entries with |want| > floor *
    max|want| (per row when 2-D); 0 when nothing qualifies."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    scale = np.abs(want).max(axis=-1, keepdims=True) if want.ndim > 1 else np.abs(want).max(initial=0.0)
    ok = np.abs(want) > np.maximum(floor * scale, 0.0)
    if not ok.any():
        return 0.0
    return float((np.abs(got - want)[ok] / np.abs(want)[ok]).max())


class SampledParity:
    """O1, the FP64 oracle and the device path on the same sampled cells;
    runs=None takes the whole mesh as one run."""

    def __init__(self, wl, runs=None, threads: int | None = None):
        import os
        self.wl = wl
        self.runs = runs
        self.edge = wl.edge
        self.threads = threads or os.cpu_count() or 1
        self.grid = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
        self.oracle = Oracle()
        self._ref = None
        self._f64 = None

    # ------------------------------------------------------------ cells
    def _runs(self):
        return [None] if self.runs is None else self.runs

    def cells(self, run):
        if run is None:
            return np.arange(self.edge ** 3)
        ix, iy, iz0, iz1 = run
        return (ix * self.edge + iy) * self.edge + np.arange(iz0, iz1)

    def all_cells(self):
        return np.concatenate([self.cells(r) for r in self._runs()])

    def blocks(self, run):
        """the target blocks (2x4x4 cells, z fastest) that hold the run"""
        if run is None:
            nb = (self.edge + 1) // 2 * ((self.edge + 3) // 4) ** 2
            return 0, nb
        ix, iy, iz0, iz1 = run
        nb = (self.edge + 3) // 4
        b = ((ix // 2) * nb + iy // 4) * nb
        return b + iz0 // 4, b + (iz1 - 1) // 4 + 1

    # ------------------------------------------------------------ O1
    def reference(self):
        """O1 on every run: rays (target, source, segment, reference-order
        columns, per-ray spectrum) and the cells' FP64 rates."""
        if self._ref is not None:
            return self._ref
        wl = self.wl
        R = RefLib(wl.edge)
        R.init(wl.lunit, wl.denstonh, wl.theta, self.threads)
        R.set_mesh(*wl.fields())
        R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
        rays = {k: [] for k in ("tgt", "src", "seg", "tau", "spectra")}
        rates = []
        for run in self._runs():
            c = self.cells(run)
            R.zero_rates()
            out = R.run_range(int(c[0]), int(c[-1]) + 1, True, want=tuple(rays))
            for k in rays:
                rays[k].append(out[k])
            rates.append(R.get_rates()[:, c])
        self._ref = {k: np.concatenate(v) for k, v in rays.items()}
        self._ref["rates"] = np.concatenate(rates, axis=1)
        return self._ref

    # ------------------------------------------------------------ FP64 oracle
    def fp64(self):
        """The FP64 precision oracle on O1's rays of the sampled cells:
        columns (FP64 march) and the cells' rates (FP64 rates, sums in
        double)."""
        if self._f64 is not None:
            return self._f64
        ref = self.reference()
        t64 = self.oracle.march_f64(self.grid, self.wl.fields(), ref["seg"])
        r64 = self.oracle.photoion_f64(self.grid, self.wl.fields(), t64, ref["tgt"], ref["seg"][:, :3],
                                       ref["spectra"])
        self._f64 = {"tau": t64, "rates": r64[:, self.all_cells()]}
        return self._f64

    # ------------------------------------------------------------ device
    def device(self, pb, precision, mode=None, surrogate=None, want_rays=False):
        """The device path on the target blocks of every run: the sampled
        cells' rates (6, ncells) and, with want_rays, the rays whose target is
        a sampled cell: (emitter position, target cell (ix, iy, iz), columns)
        in the order of the device's ray buffer."""
        import torch
        from argot_b200 import _lib as L
        rates6 = torch.zeros(6 * pb.ncell, dtype=torch.float32, device=pb.device)
        pos4 = pb.emitters()[0] if want_rays else None
        src, tgt, tau = [], [], []
        groups0 = pb.groups
        try:
            for run in self._runs():
                b0, b1 = self.blocks(run)
                pb.restrict(b0, b1)
                rays, taub = pb.alloc_group_buffers()
                for g in pb.groups:
                    pb.emit(g, rays)
                    pb.march(g, rays, taub, precision)
                    if surrogate is not None:
                        pb.rates_surrogate(g, rays, taub, rates6, surrogate)
                    else:
                        pb.rates(g, rays, taub, rates6, L.RATE_EXACT_F32 if mode is None else mode)
                    if want_rays:
                        emit, t3, _ = pb.ray_table(rays, g)
                        cell = (t3[:, 0].astype(np.int64) * self.edge + t3[:, 1]) * self.edge + t3[:, 2]
                        keep = np.isin(cell, self.cells(run))
                        cols = taub[:3 * g.nray].view(3, g.nray).t().cpu().numpy()
                        src.append(pos4[emit[keep], :3])
                        tgt.append(t3[keep])
                        tau.append(cols[keep])
                del rays, taub
        finally:
            pb.groups = groups0
        torch.cuda.synchronize()
        pb.check_device_error()
        rates = rates6.view(6, -1)[:, torch.from_numpy(self.all_cells()).to(pb.device)].cpu().numpy()
        if not want_rays:
            return rates, None
        return rates, {"src": np.concatenate(src), "tgt": np.concatenate(tgt), "tau": np.concatenate(tau)}

    # ------------------------------------------------------------ comparisons
    def by_cell(self, tgt):
        """stable order of rays by target cell (the order within a cell is
        kept)"""
        cell = (tgt[:, 0].astype(np.int64) * self.edge + tgt[:, 1]) * self.edge + tgt[:, 2]
        return np.argsort(cell, kind="stable"), cell

    def same_rays(self, dev_rays):
        """per cell, the device's rays are the reference's in its order
        (emitter positions), and the reference-order columns are bit-equal"""
        ref = self.reference()
        mine, cm = self.by_cell(dev_rays["tgt"])
        theirs, ct = self.by_cell(ref["tgt"])
        same_list = (len(mine) == len(theirs) and np.array_equal(cm[mine], ct[theirs])
                     and np.array_equal(dev_rays["src"][mine], ref["src"][theirs]))
        same_tau = same_list and np.array_equal(dev_rays["tau"][mine], ref["tau"][theirs])
        return same_list, same_tau

    def column_error_vs_f64(self, dev_rays):
        """largest relative error of the device's columns against the FP64
        march of the same rays (every positive column)"""
        ref = self.reference()
        mine, _ = self.by_cell(dev_rays["tgt"])
        theirs, _ = self.by_cell(ref["tgt"])
        t64 = self.fp64()["tau"][theirs]
        return rel_err(dev_rays["tau"][mine], t64)

    def rate_errors(self, got, want):
        """per output field, the largest relative error over the sampled
        cells with a positive rate"""
        return {n: rel_err(got[j], want[j]) for j, n in enumerate(NAMES)}
