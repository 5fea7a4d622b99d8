"""Host-side drop-in routine accum_optical_depth (no GPU needed) against the
reference's accum_optical_depth on one rank."""
import ctypes as C

import numpy as np

from conftest import ref_lib


def test_accum_optical_depth_matches_reference():
    from argot_b200 import _lib as L, abi
    lib = L.load()
    rng = np.random.default_rng(9)
    nray, nseg = 700, 650
    ray_indx = rng.permutation(nray)[:nseg].astype(np.uint64)
    tau = rng.random((nseg, 3)).astype(np.float32)
    seg = np.zeros(nseg, dtype=np.dtype(abi.RaySegment))
    seg["ray_indx"] = ray_indx
    seg["optical_depth_HI"], seg["optical_depth_HeI"], seg["optical_depth_HeII"] = tau.T
    rays = np.zeros(nray, dtype=np.dtype(abi.LightRay))
    rays["optical_depth_HI"] = 5.0
    run = abi.RunParam()
    run.nray, run.nseg, run.mpi_rank = nray, nseg, 0
    lib.accum_optical_depth(rays.ctypes.data, seg.ctypes.data, C.addressof(run), None)
    assert lib.argot_b200_last_error() == 0
    got = np.stack([rays["optical_depth_HI"], rays["optical_depth_HeI"], rays["optical_depth_HeII"]], 1)
    R = ref_lib(16)
    R.init(1.0, 1.0, 0.5, 1)
    want = R.accum_segments(nray, ray_indx, tau)
    assert np.array_equal(got, want)
