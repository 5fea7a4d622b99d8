"""Helpers of the flag-set tests: the library built for one of ARGOT's other
flag sets (argot_b200/build.py FLAGSETS), the reference's own C built with
the same flags (oracle/build.py build_ref_flags, driver
oracle/ref_flags_driver.c) and seeded cases in the reference's structs."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT

EDGE = 16
LUNIT = 6.6e-3 * 3.0856e24   # 6.6 kpc in cm (the benchmark's box)
DENSTONH = 1.0e-3            # n_H of a unit code density [cm^-3]

_LIBS = {}
_REFS = {}


def layout(tag):
    from argot_b200 import abi
    he, h2, _, _ = abi.FLAGSETS[tag]
    return abi.make_layout(he, h2)


def variant_lib(tag):
    """libargot_b200_<tag>.so (fails loudly when it is missing)."""
    if tag not in _LIBS:
        path = os.path.join(ROOT, "argot_b200", f"libargot_b200_{tag}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (python -m argot_b200.build)")
        lib = C.CDLL(path)
        vp = C.c_void_p
        for name, n in (("calc_optical_depth_cuda", 4), ("zero_out_photoion_rate_cuda", 3),
                        ("calc_photoion_rate_cuda", 5), ("smooth_photoion_rate", 5),
                        ("accum_optical_depth", 4)):
            f = getattr(lib, name)
            f.restype = None
            f.argtypes = [vp] * n
        lib.argot_b200_last_error.restype = C.c_int
        lib.argot_b200_flagset.restype = C.c_char_p
        lib.argot_b200_struct_sizes.argtypes = [vp]
        lib.argot_b200_set_dropin_march_mode.argtypes = [C.c_int]
        _LIBS[tag] = lib
    return _LIBS[tag]


def ref_flags(tag):
    """ARGOT's C built with the flag set, or skip when neither the prebuilt
    library nor the reference sources are present."""
    from oracle import build
    path = build.ref_flags_lib_path(tag, EDGE)
    if not os.path.exists(path):
        if not build.reference_available():
            pytest.skip("reference build unavailable")
        build.build_ref_flags(tag, EDGE)
    if tag not in _REFS:
        R = C.CDLL(path)
        vp = C.c_void_p
        R.refv_init.argtypes = [C.c_double, C.c_double, C.c_float, C.c_int]
        R.refv_run.restype = vp
        R.refv_mesh.restype = vp
        R.refv_photon_rate.argtypes = [C.c_int, C.c_float, C.c_double, vp]
        for name, n in (("calc_optical_depth", 3), ("calc_photoion_rate", 3), ("zero_out_photoion_rate", 2)):
            getattr(R, name).restype = None
            getattr(R, name).argtypes = [vp] * n
        _REFS[tag] = R
    return _REFS[tag]


def struct_array(Lay, name, n):
    return np.zeros(n, dtype=np.dtype(getattr(Lay, name)))


class Case:
    """One seeded problem on an EDGE^3 unit-box mesh in the flag set's
    structs: the reference's run_param (its own tables), a mesh, segments
    and light rays."""

    def __init__(self, tag, seed=1, nseg=4000, nray=3000):
        from argot_b200 import abi
        self.tag = tag
        he, h2, pc, cosmo = abi.FLAGSETS[tag]
        self.he, self.h2 = he, h2
        self.Lay = Lay = layout(tag)
        R = self.R = ref_flags(tag)
        self.anow = 0.5 if cosmo else 1.0
        assert R.refv_init(LUNIT, DENSTONH, self.anow, 1) == 0
        ncell = EDGE ** 3
        self.ncell = ncell
        rng = np.random.default_rng(seed)
        # the reference's mesh, viewed in place
        buf = (C.c_char * (ncell * C.sizeof(Lay.FluidMesh))).from_address(R.refv_mesh())
        self.mesh_ref = np.frombuffer(buf, dtype=np.dtype(Lay.FluidMesh))
        m = np.zeros(ncell, dtype=np.dtype(Lay.FluidMesh))
        m["dens"] = np.exp(rng.normal(0.0, 1.0, ncell)).astype(np.float32)
        xi = rng.uniform(1e-4, 0.3, ncell).astype(np.float32)
        m["chem"]["fHI"] = 1.0 - xi
        m["chem"]["fHII"] = xi
        if he:
            m["chem"]["fHeII"] = rng.uniform(1e-4, 0.2, ncell).astype(np.float32)
            m["chem"]["fHeI"] = 1.0 - m["chem"]["fHeII"]
        if h2:
            for k, (lo, hi) in (("fHM", (1e-9, 1e-6)), ("fH2I", (1e-6, 1e-2)), ("fH2II", (1e-9, 1e-6))):
                m["chem"][k] = np.exp(rng.uniform(np.log(lo), np.log(hi), ncell)).astype(np.float32)
        self.mesh_ref[:] = m
        self.mesh_init = m
        self.run_ptr = R.refv_run()
        # segments anywhere in the box
        seg = struct_array(Lay, "RaySegment", nseg)
        seg["ray_indx"] = np.arange(nseg)
        p = rng.uniform(0.0, 1.0, (nseg, 6)).astype(np.float32)
        for i, k in enumerate(("xpos_start", "ypos_start", "zpos_start", "xpos_end", "ypos_end", "zpos_end")):
            seg[k] = p[:, i]
        self.seg = seg
        # light rays: a few sources, targets in runs per cell (the order the
        # reference emits), columns from thin to thick
        nsrc = 8
        spos = rng.uniform(0.0, 1.0, (nsrc, 3)).astype(np.float32)
        spec = np.zeros((nsrc, 256))
        for s in range(nsrc):
            R.refv_photon_rate(0, C.c_float(1.0e5), 10.0 ** rng.uniform(48, 50), spec[s].ctypes.data)
        tgt_cells = np.sort(rng.integers(0, ncell, nray))
        ray = struct_array(Lay, "LightRay", nray)
        which = rng.integers(0, nsrc, nray)
        ray["src"]["type"] = 0
        ray["src"]["param"] = 1.0e5
        ray["src"]["xpos"] = spos[which, 0]
        ray["src"]["ypos"] = spos[which, 1]
        ray["src"]["zpos"] = spos[which, 2]
        ray["src"]["photon_rate"] = spec[which]
        ray["ix_target"] = tgt_cells // (EDGE * EDGE)
        ray["iy_target"] = (tgt_cells // EDGE) % EDGE
        ray["iz_target"] = tgt_cells % EDGE
        # no ray starts inside its own target cell (whose entry column the
        # reference would make negative)
        src_cell = (np.floor(spos * EDGE).astype(np.int64) @ np.array([EDGE * EDGE, EDGE, 1]))[which]
        ray = ray[src_cell != tgt_cells]
        # the columns as ARGOT forms them: the reference's march from the
        # source to the target cell's centre (calc_ray_segment.c:47-126)
        d = np.float64(np.float32(1.0) / np.float32(EDGE))
        seg = struct_array(Lay, "RaySegment", len(ray))
        seg["xpos_start"], seg["ypos_start"], seg["zpos_start"] = (ray["src"][k] for k in ("xpos", "ypos", "zpos"))
        for a in ("x", "y", "z"):
            seg[a + "pos_end"] = ((ray[f"i{a}_target"].astype(np.float32).astype(np.float64) + 0.5) * d).astype(np.float32)
        run = self.run_bytes(nseg=len(seg))
        C.memmove(self.run_ptr, C.addressof(run), C.sizeof(run))
        R.calc_optical_depth(seg.ctypes.data, self.mesh_ref.ctypes.data, self.run_ptr)
        for c in Lay.columns:
            ray["optical_depth_" + c] = seg["optical_depth_" + c]
        self.ray = ray

    def run_bytes(self, nseg=0, nray=0):
        """a copy of the reference's run_param with the counts set"""
        r = self.Lay.RunParam()
        C.memmove(C.addressof(r), self.run_ptr, C.sizeof(r))
        r.nseg, r.nray = nseg, nray
        return r

    def rates_of(self, mesh):
        return np.stack([mesh["prev_chem"][k] for k in self.Lay.rates], 1)
