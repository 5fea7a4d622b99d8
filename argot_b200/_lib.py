"""ctypes binding of libargot_b200.so (the C ABI in include/argot_b200.h).

The library is built in-tree (``argot_b200/build.py``); the environment
variable ARGOT_B200_LIB may name another build of it.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libargot_b200.so")

OK = 0
EINVAL, ECUDA, ENOMEM, EDEVICE, ENOTSUP = -1, -2, -3, -4, -5

PRECISION_REFERENCE = 0
PRECISION_KAHAN = 1
RATE_EXACT_F64 = 0
RATE_EXACT_F32 = 1
RATE_SURROGATE = 2

# Every function the header declares (name -> (restype, argtypes)).
vp, u64, u32, i32, f32, f64 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_float, C.c_double


class Grid(C.Structure):
    """argot_b200_grid"""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("ix0", C.c_int), ("iy0", C.c_int), ("iz0", C.c_int),
                ("xmin", C.c_float), ("ymin", C.c_float), ("zmin", C.c_float),
                ("xmax", C.c_float), ("ymax", C.c_float), ("zmax", C.c_float),
                ("xmin_local", C.c_float), ("ymin_local", C.c_float), ("zmin_local", C.c_float),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
                ("lunit", C.c_double), ("denstonh", C.c_double)]


GP = C.POINTER(Grid)


class BatchProblem(C.Structure):
    """argot_b200_batch_problem"""
    _fields_ = [("grid", Grid), ("packed_dev", C.c_void_p), ("tree", C.c_void_p),
                ("blk_offsets_dev", C.c_void_p), ("blk_offsets_host", C.c_void_p),
                ("rays_dev", C.c_void_p), ("rates6_dev", C.c_void_p)]


class BatchConfig(C.Structure):
    """argot_b200_batch_config"""
    _fields_ = [("warps_per_cta", C.c_int), ("ctas_per_sm", C.c_int), ("blocks_per_item", C.c_int),
                ("order", C.c_int), ("mode", C.c_int), ("parts", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

SIGNATURES = {
    "argot_b200_last_error": (i32, []),
    "argot_b200_error_string": (C.c_char_p, [i32]),
    "argot_b200_version": (C.c_char_p, []),
    "argot_b200_flagset": (C.c_char_p, []),
    "argot_b200_dev_tree_build": (i32, [vp, i32, vp, vp, f32, vp, vp]),
    "argot_b200_dev_tree_info": (i32, [vp, vp, vp, vp]),
    "argot_b200_dev_tree_copy": (i32, [vp, vp, vp, vp, vp, vp]),
    "argot_b200_struct_sizes": (None, [vp]),
    "argot_b200_abi_check": (i32, [vp, i32]),
    "calc_optical_depth_cuda": (None, [vp, vp, vp, vp]),
    "calc_photoion_rate_cuda": (None, [vp, vp, vp, vp, vp]),
    "zero_out_photoion_rate_cuda": (None, [vp, vp, vp]),
    "accum_optical_depth": (None, [vp, vp, vp, vp]),
    "argot_b200_set_dropin_march_mode": (i32, [i32]),
    "smooth_photoion_rate": (None, [vp, vp, vp, vp, vp]),
    "calc_diffuse_photon_radiation": (None, [vp, vp, vp, vp, vp, vp, vp]),
    "argot_b200_run_group": (i32, [GP, vp, vp, u64, u64, vp, vp, u64, vp, vp, i32, i32, i32, i32, vp, vp, vp]),
    "argot_b200_art_angle_table": (i32, [i32, vp, vp, vp]),
    "argot_b200_art_step_factors": (None, [vp]),
    "argot_b200_art_create": (i32, [vp, vp, i32, vp, vp]),
    "argot_b200_art_destroy": (None, [vp]),
    "argot_b200_art_num_angles": (i32, [vp]),
    "argot_b200_art_workspace": (u64, [GP, i32]),
    "argot_b200_art_rates": (i32, [vp, GP, f64, vp, vp, vp, i32, vp, vp]),
    "argot_b200_set_dropin_smooth_faces": (i32, [i32]),
    "argot_b200_pack_fields": (i32, [GP, vp, vp, vp, vp, vp, vp]),
    "argot_b200_pack_fluid_mesh": (i32, [GP, vp, vp, vp]),
    "argot_b200_tree_build": (i32, [GP, i32, vp, vp, f32, C.POINTER(vp)]),
    "argot_b200_tree_free": (None, [vp]),
    "argot_b200_tree_num_emitters": (i32, [vp]),
    "argot_b200_tree_num_nodes": (i32, [vp]),
    "argot_b200_tree_emitters": (i32, [vp, vp, vp]),
    "argot_b200_dev_tree_upload": (i32, [vp, C.POINTER(vp), vp]),
    "argot_b200_dev_tree_free": (None, [vp]),
    "argot_b200_num_blocks": (i32, [GP, C.POINTER(u64)]),
    "argot_b200_count_rays": (i32, [GP, vp, u64, u64, vp, vp, vp]),
    "argot_b200_scan_blocks": (i32, [vp, u64, u64, vp, C.POINTER(u64), vp]),
    "argot_b200_scan_blocks_static": (i32, [vp, u64, u64, vp, C.POINTER(u64), vp]),
    "argot_b200_emit_rays": (i32, [GP, vp, u64, u64, vp, u64, vp, vp]),
    "argot_b200_march_rays": (i32, [GP, vp, vp, u64, u64, vp, u64, vp, u64, vp, i32, vp, vp]),
    "argot_b200_march_segments": (i32, [GP, vp, u64, vp, vp, i32, vp]),
    "argot_b200_stitch": (i32, [u64, vp, vp, u64, vp, vp]),
    "argot_b200_photoion_rays": (i32, [GP, vp, vp, u64, u64, vp, u64, vp, u64, vp, i32, vp, vp]),
    "argot_b200_check_device_error": (i32, [vp]),
    "argot_b200_smooth_rates": (i32, [GP, vp, vp, i32, vp]),
    "argot_b200_tables": (None, [vp, vp]),
    "argot_b200_photon_rate": (None, [i32, f32, f64, vp]),
    "argot_b200_photon_counts": (None, [i32, f32, vp, vp]),
    "argot_b200_dev_tree_set_blackbody": (i32, [vp, vp, vp, vp]),
    "argot_b200_mlp_num_params": (i32, []),
    "argot_b200_mlp_spectra": (i32, [i32, vp, vp]),
    "argot_b200_mlp_samples": (i32, [vp, vp, i32, u64, u64, vp, vp, vp]),
    "argot_b200_mlp_workspace": (u64, [i32]),
    "argot_b200_mlp_forward": (i32, [vp, vp, i32, vp, vp]),
    "argot_b200_mlp_train_step": (i32, [vp, vp, vp, vp, vp, i32, f32, i32, vp, vp, vp, vp]),
    "argot_b200_surrogate_create": (i32, [vp, vp, f32, C.POINTER(vp)]),
    "argot_b200_surrogate_free": (None, [vp]),
    "argot_b200_surrogate_eval": (i32, [vp, vp, i32, vp, vp]),
    "argot_b200_surrogate_workspace": (u64, [u64]),
    "argot_b200_batch_create": (i32, [C.POINTER(BatchProblem), i32, C.POINTER(vp)]),
    "argot_b200_batch_free": (None, [vp]),
    "argot_b200_batch_configure": (i32, [vp, C.POINTER(BatchConfig)]),
    "argot_b200_batch_get_config": (i32, [vp, C.POINTER(BatchConfig)]),
    "argot_b200_batch_num_items": (i32, [vp]),
    "argot_b200_batch_run": (i32, [vp, vp, vp]),
    "argot_b200_batch_graph_launch": (i32, [vp, vp]),
    "argot_b200_batch_tune": (i32, [vp, i32, C.POINTER(BatchConfig), C.POINTER(f32), vp]),
    "argot_b200_photoion_rays_surrogate": (i32, [GP, vp, vp, vp, u64, u64, vp, u64, vp, u64, vp, vp, vp,
                                                 vp, vp]),
}

_lock = threading.Lock()
_lib = None


class ArgotError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = _lib.argot_b200_error_string(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: {msg} ({code})")


def load(path: str | None = None):
    """Loads (once) and returns the library; raises if it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = path or os.environ.get("ARGOT_B200_LIB") or LIB_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is not built; run `python -m argot_b200.build` (no CPU fallback exists)")
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int, where: str):
    if rc != OK:
        raise ArgotError(rc, where)


def exported_symbols():
    return list(SIGNATURES)
