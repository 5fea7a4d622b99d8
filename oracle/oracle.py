"""ctypes front-ends for the CPU checkers (test infrastructure only).

``RefLib(edge)``  ARGOT's own hot-path C (O1), built by ``oracle/build.py``.
``Oracle()``      the restatement in ``oracle/argot_oracle.c`` (ref-order FP32
                  march, FP64 precision oracle, ref-order FP64 rates, tables).

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline / reference
arm import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

NGRID_NU = 256

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OrcGrid(C.Structure):
    """Mirror of ``orc_grid`` in argot_oracle.c."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("rank_x", C.c_int), ("rank_y", C.c_int), ("rank_z", C.c_int),
                ("xmin", C.c_float), ("ymin", C.c_float), ("zmin", C.c_float),
                ("xmin_local", C.c_float), ("ymin_local", C.c_float), ("zmin_local", C.c_float),
                ("delta_x", C.c_float), ("delta_y", C.c_float), ("delta_z", C.c_float),
                ("lunit", C.c_double), ("denstonh", C.c_double)]


def unit_box_grid(edge: int, lunit: float, denstonh: float) -> OrcGrid:
    d = np.float32(np.float32(1.0) / np.float32(edge))
    return OrcGrid(edge, edge, edge, 0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                   float(d), float(d), float(d), lunit, denstonh)


class Oracle:
    """The C restatement (always buildable: needs only gcc)."""

    def __init__(self, path: str | None = None):
        path = path or _build.oracle_lib_path()
        if not os.path.exists(path):
            _build.build_oracle()
        self.lib = L = C.CDLL(path)
        L.orc_tables.argtypes = [_f64p, _f32p, _f64p]
        L.orc_photon_rate.argtypes = [C.c_int, C.c_float, C.c_double, _f64p]
        for name in ("orc_march_f32ref",):
            getattr(L, name).argtypes = [C.POINTER(OrcGrid), _f32p, _f32p, _f32p, _f32p,
                                         C.c_uint64, _f32p, _f32p]
        L.orc_march_f64.argtypes = [C.POINTER(OrcGrid), _f32p, _f32p, _f32p, _f32p,
                                    C.c_uint64, _f32p, _f64p]
        L.orc_count_crossings.argtypes = [C.POINTER(OrcGrid), C.c_uint64, _f32p, _u64p]
        L.orc_accum.argtypes = [C.c_uint64, C.c_uint64, _u64p, _f32p, _f32p]
        L.orc_photoion_f64ref.argtypes = [C.POINTER(OrcGrid), _f32p, _f32p, _f32p, _f32p,
                                          _f64p, _f32p, C.c_uint64, _f32p, _i32p, _f32p,
                                          _f64p, C.c_void_p, _f32p]
        L.orc_photoion_f64.argtypes = [C.POINTER(OrcGrid), _f32p, _f32p, _f32p, _f32p,
                                       _f64p, _f32p, C.c_uint64, _f64p, _i32p, _f32p,
                                       _f64p, C.c_void_p, _f64p]
        L.orc_photoion_f64ref_per_ray.argtypes = [C.POINTER(OrcGrid), _f32p, _f32p, _f32p,
                                                  _f32p, _f64p, _f32p, C.c_uint64, _f32p,
                                                  _i32p, _f32p, _f64p, C.c_void_p, _f64p]

    def tables(self):
        nu = np.zeros(NGRID_NU, np.float64)
        cs = np.zeros((NGRID_NU, 3), np.float32)
        meta = np.zeros(3, np.float64)
        self.lib.orc_tables(nu, cs, meta)
        return nu, cs, meta

    def photon_rate(self, typ: int, param: float, total: float):
        out = np.zeros(NGRID_NU, np.float64)
        self.lib.orc_photon_rate(int(typ), float(param), float(total), out)
        return out

    def march_f32ref(self, grid, fields, pos6):
        pos6 = np.ascontiguousarray(pos6, np.float32)
        n = pos6.shape[0]
        tau = np.zeros((n, 3), np.float32)
        self.lib.orc_march_f32ref(C.byref(grid), *fields, n, pos6, tau)
        return tau

    def march_f64(self, grid, fields, pos6):
        pos6 = np.ascontiguousarray(pos6, np.float32)
        n = pos6.shape[0]
        tau = np.zeros((n, 3), np.float64)
        self.lib.orc_march_f64(C.byref(grid), *fields, n, pos6, tau)
        return tau

    def count_crossings(self, grid, pos6):
        pos6 = np.ascontiguousarray(pos6, np.float32)
        out = np.zeros(pos6.shape[0], np.uint64)
        self.lib.orc_count_crossings(C.byref(grid), pos6.shape[0], pos6, out)
        return out

    def accum(self, nray, ray_indx, seg_tau):
        out = np.zeros((nray, 3), np.float32)
        self.lib.orc_accum(nray, len(ray_indx), np.ascontiguousarray(ray_indx, np.uint64),
                           np.ascontiguousarray(seg_tau, np.float32), out)
        return out

    def photoion_f64ref(self, grid, fields, tau3, tgt3, src3, spectra, spec_index=None,
                        rates6=None):
        ncell = grid.nx * grid.ny * grid.nz
        if rates6 is None:
            rates6 = np.zeros((6, ncell), np.float32)
        si = None if spec_index is None else np.ascontiguousarray(spec_index, np.uint64)
        nu, cs, _ = self.tables()
        self.lib.orc_photoion_f64ref(C.byref(grid), *fields, nu, cs, len(tau3),
                                     np.ascontiguousarray(tau3, np.float32),
                                     np.ascontiguousarray(tgt3, np.int32),
                                     np.ascontiguousarray(src3, np.float32),
                                     np.ascontiguousarray(spectra, np.float64), _vp(si), rates6)
        return rates6

    def photoion_f64(self, grid, fields, tau3, tgt3, src3, spectra, spec_index=None):
        ncell = grid.nx * grid.ny * grid.nz
        rates6 = np.zeros((6, ncell), np.float64)
        si = None if spec_index is None else np.ascontiguousarray(spec_index, np.uint64)
        nu, cs, _ = self.tables()
        self.lib.orc_photoion_f64(C.byref(grid), *fields, nu, cs, len(tau3),
                                  np.ascontiguousarray(tau3, np.float64),
                                  np.ascontiguousarray(tgt3, np.int32),
                                  np.ascontiguousarray(src3, np.float32),
                                  np.ascontiguousarray(spectra, np.float64), _vp(si), rates6)
        return rates6

    def photoion_f64ref_per_ray(self, grid, fields, tau3, tgt3, src3, spectra,
                                spec_index=None):
        out = np.zeros((len(tau3), 6), np.float64)
        si = None if spec_index is None else np.ascontiguousarray(spec_index, np.uint64)
        nu, cs, _ = self.tables()
        self.lib.orc_photoion_f64ref_per_ray(C.byref(grid), *fields, nu, cs, len(tau3),
                                             np.ascontiguousarray(tau3, np.float32),
                                             np.ascontiguousarray(tgt3, np.int32),
                                             np.ascontiguousarray(src3, np.float32),
                                             np.ascontiguousarray(spectra, np.float64),
                                             _vp(si), out)
        return out


class RefLib:
    """ARGOT's own C for an N^3 single-rank mesh (O1)."""

    _cache: dict = {}

    def __init__(self, edge: int, fast_math: bool = False, isolated: bool = False, path: str = None):
        if path is None:
            path = _build.ref_lib_path(edge, fast_math, isolated)
            if not os.path.exists(path):
                if not _build.reference_available():
                    raise FileNotFoundError(f"{path} missing and the reference is absent")
                _build.build_ref(edge, fast_math=fast_math, isolated=isolated)
        # each edge is a distinct library with its own static state
        self.lib = L = C.CDLL(path, mode=C.RTLD_LOCAL)
        self.edge = edge
        L.ref_mesh_edge.restype = C.c_int
        L.ref_struct_sizes.argtypes = [_u64p]
        L.ref_struct_offsets.argtypes = [_u64p]
        L.ref_init.argtypes = [C.c_double, C.c_double, C.c_float, C.c_int]
        L.ref_init.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_tables.argtypes = [_f64p, _f32p, _f64p]
        L.ref_photon_rate.argtypes = [C.c_int, C.c_float, C.c_double, _f64p]
        L.ref_set_mesh.argtypes = [_f32p, _f32p, _f32p, _f32p]
        L.ref_get_rates.argtypes = [_f32p]
        L.ref_set_sources.argtypes = [C.c_int, _i32p, _f32p, _f32p, _f64p, C.c_int]
        L.ref_set_sources.restype = C.c_int
        L.ref_get_source_spectra.argtypes = [_f64p]
        L.ref_count_rays.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.ref_count_rays.restype = C.c_uint64
        L.ref_run_range.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 7
        L.ref_run_range.restype = C.c_int64
        L.ref_march_segments.argtypes = [C.c_uint64, _f32p, _f32p, C.c_void_p]
        L.ref_accum_segments.argtypes = [C.c_uint64, C.c_uint64, _u64p, _f32p, _f32p]
        L.ref_photoion_rays.argtypes = [C.c_uint64, _i32p, _f32p, _f64p, _f32p, C.c_void_p]
        L.ref_smooth_rates.argtypes = [_f32p]
        L.ref_write_files.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_read_files.argtypes = [C.c_char_p, C.c_char_p, _f32p, _f32p, _f32p, _f32p, _i32p, _f32p,
                                     _f32p, _f64p, C.c_int64]
        L.ref_read_files.restype = C.c_int64
        L.ref_art_init.argtypes = [C.c_double]
        L.ref_art_init.restype = C.c_int
        L.ref_art_table.argtypes = [_f32p, _i32p, _i32p, _f32p]
        L.ref_art_set_mesh.argtypes = [_f32p]
        L.ref_art_run.argtypes = [_f32p]
        L.ref_art_run.restype = C.c_double
        assert L.ref_mesh_edge() == edge
        self.isolated = isolated

    def struct_sizes(self):
        out = np.zeros(10, np.uint64)
        self.lib.ref_struct_sizes(out)
        return out

    def struct_offsets(self):
        out = np.zeros(40, np.uint64)
        self.lib.ref_struct_offsets(out)
        return out[:32]

    def write_files(self, mesh_file: str, src_prefix: str):
        """The reference's output_mesh_single / output_src on the loaded
        mesh and sources."""
        self.lib.ref_write_files(mesh_file.encode(), src_prefix.encode())

    def read_files(self, mesh_file: str, src_file: str, max_src: int = 1 << 16):
        """The reference's input_mesh_single / input_src_file: (dens, fHI,
        fHeI, fHeII), (type, param, xyz, photon rates)."""
        n = self.edge ** 3
        f = [np.zeros(n, np.float32) for _ in range(4)]
        typ = np.zeros(max_src, np.int32)
        par = np.zeros(max_src, np.float32)
        xyz = np.zeros((max_src, 3), np.float32)
        spec = np.zeros((max_src, NGRID_NU), np.float64)
        k = self.lib.ref_read_files(mesh_file.encode(), src_file.encode(), *f, typ, par, xyz, spec, max_src)
        assert k >= 0
        return f, (typ[:k], par[:k], xyz[:k], spec[:k])

    def smooth_rates(self, rates6):
        """smooth_photoion_rate.c on six rate planes (6, ncell) float32;
        returns the smoothed planes (needs init() first)."""
        r = np.ascontiguousarray(rates6, np.float32).reshape(6, -1).copy()
        self.lib.ref_smooth_rates(r)
        return r

    def init(self, lunit, denstonh, theta=0.5, nthreads=1):
        assert self.lib.ref_init(lunit, denstonh, theta, nthreads) == 0

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def tables(self):
        nu = np.zeros(NGRID_NU, np.float64)
        cs = np.zeros((NGRID_NU, 3), np.float32)
        meta = np.zeros(3, np.float64)
        self.lib.ref_tables(nu, cs, meta)
        return nu, cs, meta

    def photon_rate(self, typ, param, total):
        out = np.zeros(NGRID_NU, np.float64)
        self.lib.ref_photon_rate(int(typ), float(param), float(total), out)
        return out

    def set_mesh(self, dens, fHI, fHeI, fHeII):
        self.lib.ref_set_mesh(*(np.ascontiguousarray(a, np.float32).ravel()
                                for a in (dens, fHI, fHeI, fHeII)))

    def set_sources(self, typ, param, xyz, total, build_tree=True):
        n = len(typ)
        r = self.lib.ref_set_sources(n, np.ascontiguousarray(typ, np.int32),
                                     np.ascontiguousarray(param, np.float32),
                                     np.ascontiguousarray(xyz, np.float32).ravel(),
                                     np.ascontiguousarray(total, np.float64), int(build_tree))
        assert r == 0, r
        self.nsrc = n

    def source_spectra(self):
        out = np.zeros((self.nsrc, NGRID_NU), np.float64)
        self.lib.ref_get_source_spectra(out)
        return out

    def count_rays(self, im0, im1, per_cell=False):
        if per_cell:
            pc = np.zeros(im1 - im0, np.uint64)
            tot = self.lib.ref_count_rays(im0, im1, _vp(pc))
            return tot, pc
        return self.lib.ref_count_rays(im0, im1, None)

    def zero_rates(self):
        self.lib.ref_zero_rates()

    def get_rates(self):
        out = np.zeros((6, self.edge ** 3), np.float32)
        self.lib.ref_get_rates(out)
        return out

    def run_range(self, im0, im1, do_photo=True, want=("tgt", "src", "seg", "tau")):
        nray = self.count_rays(im0, im1)
        tgt = np.zeros((nray, 3), np.int32) if "tgt" in want else None
        src = np.zeros((nray, 3), np.float32) if "src" in want else None
        seg = np.zeros((nray, 6), np.float32) if "seg" in want else None
        tau = np.zeros((nray, 3), np.float32) if "tau" in want else None
        ssum = np.zeros(nray, np.float64) if "spec_sum" in want else None
        spectra = np.zeros((nray, NGRID_NU), np.float64) if "spectra" in want else None
        times = np.zeros(4, np.float64)
        n = self.lib.ref_run_range(im0, im1, int(do_photo), _vp(tgt), _vp(src), _vp(seg),
                                   _vp(tau), _vp(ssum), _vp(spectra), _vp(times))
        assert n == nray, (n, nray)
        return dict(tgt=tgt, src=src, seg=seg, tau=tau, spec_sum=ssum, spectra=spectra,
                    times=times, nray=nray)

    # ---- ART diffuse radiation (src/diffuse_photon, CPU build)
    def art_init(self, uenetok):
        """setup_diffuse_photon: the angle table and step-function factors;
        returns the number of angles (12 N_SIDE^2)"""
        self.n_ang = int(self.lib.ref_art_init(float(uenetok)))
        return self.n_ang

    def art_table(self):
        n = self.n_ang
        d = np.zeros((n, 3), np.float32)
        bc = np.zeros((n, 2), np.int32)
        c8 = np.zeros(8, np.int32)
        st = np.zeros(6, np.float32)
        self.lib.ref_art_table(d, bc, c8, st)
        return d, bc, c8, st

    def art_set_mesh(self, planes8):
        """dens, fHI, fHII, fHeI, fHeII, fHeIII, felec, prev_uene"""
        self.lib.ref_art_set_mesh(np.ascontiguousarray(planes8, np.float32).reshape(8, -1))

    def art_run(self):
        """calc_diffuse_photon_radiation: the six diffuse rate planes and the
        wall time"""
        out = np.zeros((6, self.edge ** 3), np.float32)
        t = self.lib.ref_art_run(out)
        return out, t

    def march_segments(self, pos6):
        pos6 = np.ascontiguousarray(pos6, np.float32)
        tau = np.zeros((pos6.shape[0], 3), np.float32)
        wall = C.c_double()
        self.lib.ref_march_segments(pos6.shape[0], pos6, tau, C.byref(wall))
        return tau, wall.value

    def accum_segments(self, nray, ray_indx, seg_tau):
        out = np.zeros((nray, 3), np.float32)
        self.lib.ref_accum_segments(nray, len(ray_indx),
                                    np.ascontiguousarray(ray_indx, np.uint64),
                                    np.ascontiguousarray(seg_tau, np.float32), out)
        return out

    def photoion_rays(self, tgt3, src3, spectra, tau3):
        wall = C.c_double()
        self.lib.ref_photoion_rays(len(tgt3), np.ascontiguousarray(tgt3, np.int32),
                                   np.ascontiguousarray(src3, np.float32),
                                   np.ascontiguousarray(spectra, np.float64),
                                   np.ascontiguousarray(tau3, np.float32), C.byref(wall))
        return wall.value


class RefGpu(RefLib):
    """ARGOT's own GPU entry points (calc_optical_depth_cuda,
    calc_photoion_rate_cuda, zero_out_photoion_rate_cuda) compiled for
    sm_100a with the reference's nvcc flags, with the CPU reference that
    builds their rays (``oracle/ref_gpu_driver.cu``).  Needs a GPU."""

    def __init__(self, edge: int):
        path = _build.refgpu_lib_path(edge)
        if not os.path.exists(path):
            if not _build.reference_available():
                raise FileNotFoundError(f"{path} missing and the reference is absent")
            _build.build_ref_gpu(edge)
        super().__init__(edge, path=path)
        L = self.lib
        L.refgpu_edge.restype = C.c_int
        L.refgpu_init.restype = C.c_int
        L.refgpu_zero_rates.restype = C.c_int
        L.refgpu_get_rates.argtypes = [_f32p]
        L.refgpu_get_rates.restype = C.c_int
        L.refgpu_run_range.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64,
                                       _f64p]
        L.refgpu_run_range.restype = C.c_int
        L.refgpu_use_entry_points.argtypes = [C.c_void_p, C.c_void_p]
        assert L.refgpu_edge() == edge

    def use_entry_points(self, lib=None):
        """run the group loop with another library's calc_optical_depth_cuda
        and calc_photoion_rate_cuda (a drop-in), or the reference's own
        (lib None)"""
        if lib is None:
            self.lib.refgpu_use_entry_points(None, None)
        else:
            self.lib.refgpu_use_entry_points(C.cast(lib.calc_optical_depth_cuda, C.c_void_p),
                                             C.cast(lib.calc_photoion_rate_cuda, C.c_void_p))

    def upload(self):
        """mesh and run parameters to the device (after set_mesh and
        set_sources)"""
        rc = self.lib.refgpu_init()
        assert rc == 0, f"refgpu_init: {rc}"

    def zero_rates_gpu(self):
        assert self.lib.refgpu_zero_rates() == 0

    def rates_gpu(self):
        out = np.zeros((6, self.edge ** 3), np.float32)
        assert self.lib.refgpu_get_rates(out) == 0
        return out

    def run_range_gpu(self, im0, im1, kernel_reps=0, want=()):
        """the reference's GPU path over target cells [im0, im1); returns the
        counts and timings of refgpu_run_range (and the segment end points
        and stitched columns when asked)"""
        nray = self.count_rays(im0, im1)
        seg = np.zeros((nray, 6), np.float32) if "seg" in want else None
        tau = np.zeros((nray, 3), np.float32) if "tau" in want else None
        out = np.zeros(10, np.float64)
        rc = self.lib.refgpu_run_range(im0, im1, int(kernel_reps), _vp(seg), _vp(tau), nray, out)
        assert rc == 0, f"refgpu_run_range: {rc}"
        return dict(nray=int(out[0]), nseg=int(out[1]), setup_s=out[2], march_s=out[3], accum_s=out[4],
                    rates_s=out[5], march_kernel_ms=out[6], rate_kernel_ms=out[7], groups=int(out[8]),
                    seg=seg, tau=tau)

    def close(self):
        self.lib.refgpu_free()
