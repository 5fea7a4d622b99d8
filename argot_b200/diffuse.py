"""ART diffuse radiation on the device (ARGOT src/diffuse_photon, one rank).

The second radiative-transfer path of ARGOT: recombination photons carried
along long characteristics in 12 nside^2 HEALPix directions
(``calc_diffuse_photon_radiation.c``).  This module drives the C ABI
(``argot_b200_art_*``): the reference's angle table and step-function
factors, built on the host by the library, and one call that adds the
diffuse rates of every cell to the six rate planes.

Inputs per cell, as eight planes of float32: ``dens`` and the ``prev_chem``
fractions ``fHI, fHII, fHeI, fHeII, fHeIII, felec`` and ``prev_uene`` of
ARGOT's ``fluid_mesh``; ``uenetok`` converts ``uene`` to a temperature as in
``run_param``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

FIELDS = ("dens", "fHI", "fHII", "fHeI", "fHeII", "fHeIII", "felec", "uene")
NSIDE = 8  # the reference's N_SIDE (run_param.h:159): 768 directions


def angle_table(nside: int = NSIDE):
    """(dir3 float32 (n, 3), base_corner int32 (n, 2), per-octant counts)
    in the reference's processing order (set_angle.c)"""
    lib = L.load()
    n = 12 * nside * nside
    d = np.zeros((n, 3), np.float32)
    bc = np.zeros((n, 2), np.int32)
    c8 = np.zeros(8, np.int32)
    m = lib.argot_b200_art_angle_table(nside, d.ctypes.data, bc.ctypes.data, c8.ctypes.data)
    L.check(m if m < 0 else 0, "art_angle_table")
    return d, bc, c8


def step_factors():
    """set_step_func_factor: ionisation and heating factors of HI, HeI, HeII"""
    out = np.zeros(6, np.float32)
    L.load().argot_b200_art_step_factors(out.ctypes.data)
    return out


class Diffuse:
    """A direction set on the current device and the call that adds the
    diffuse rates (argot_b200_art_rates)."""

    def __init__(self, nside: int = NSIDE, table=None):
        self.lib = L.load()
        d, bc, _ = table if table is not None else angle_table(nside)
        d = np.ascontiguousarray(d, np.float32)
        bc = np.ascontiguousarray(bc, np.int32)
        st = step_factors()
        h = C.c_void_p()
        L.check(self.lib.argot_b200_art_create(d.ctypes.data, bc.ctypes.data, len(d), st.ctypes.data,
                                               C.byref(h)), "art_create")
        self.h = h
        self.nang = len(d)
        self._work = None

    def close(self):
        if self.h:
            self.lib.argot_b200_art_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def default_pass(self, grid, budget_bytes: int = 2 << 30) -> int:
        """angles per pass: about a million rays in flight, accumulators
        within budget_bytes"""
        n = grid.nx * grid.ny * grid.nz
        face = max(grid.nx * grid.ny, grid.ny * grid.nz, grid.nz * grid.nx)
        a = max(1, min(self.nang, (1 << 20) // face))
        return int(max(1, min(a, budget_bytes // (16 * n))))

    def rates(self, grid, uenetok: float, fields8, rates6, angles_per_pass: int | None = None,
              crossings=None, stream=None):
        """Adds the diffuse rates to rates6 (torch float32 on the device, six
        planes); fields8: torch float32 (8, ncell) on the device."""
        import torch
        a = angles_per_pass or self.default_pass(grid)
        need = int(self.lib.argot_b200_art_workspace(C.byref(grid), a))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.uint8, device=rates6.device)
        st = stream if stream is not None else torch.cuda.current_stream(rates6.device).cuda_stream
        L.check(self.lib.argot_b200_art_rates(self.h, C.byref(grid), float(uenetok), fields8.data_ptr(),
                                              rates6.data_ptr(), self._work.data_ptr(), a,
                                              crossings.data_ptr() if crossings is not None else None, st),
                "art_rates")
