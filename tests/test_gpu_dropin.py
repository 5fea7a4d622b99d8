"""The reference-signature entry points (calc_optical_depth_cuda,
calc_photoion_rate_cuda, zero_out_photoion_rate_cuda) driven with the
reference's own struct layouts, against the reference's results."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden, ref_lib

pytestmark = pytest.mark.gpu


def _run_param(edge, lunit, denstonh, nseg=0, nray=0):
    from argot_b200 import abi
    r = abi.RunParam()
    r.helium_flag = 1
    r.ngrid_nu = 256
    r.mpi_nproc = 1
    r.nnode_x = r.nnode_y = r.nnode_z = 1
    r.lunit, r.denstonh, r.anow = lunit, denstonh, 1.0
    r.xmin = r.ymin = r.zmin = 0.0
    r.xmax = r.ymax = r.zmax = 1.0
    r.xmin_local = r.ymin_local = r.zmin_local = 0.0
    r.xmax_local = r.ymax_local = r.zmax_local = 1.0
    for a in ("x", "y", "z"):
        setattr(r, f"nmesh_{a}_total", edge)
        setattr(r, f"nmesh_{a}_local", edge)
        setattr(r, f"delta_{a}", float(np.float32(1.0) / np.float32(edge)))
    r.nseg, r.nray = nseg, nray
    r.theta_crit = 0.5
    # the tables the caller's setup_freq_param / setup_cross_section fill
    # (source.c:38-53, cross_section.c:5-22); the drop-in reads them
    from argot_b200 import _lib as L
    nu = np.zeros(256)
    cs3 = np.zeros(3 * 256, np.float32)
    L.load().argot_b200_tables(nu.ctypes.data, cs3.ctypes.data)
    r.freq.log_nu_min, r.freq.log_nu_max, r.freq.dlog_nu = 0.0, 1.5, 1.5 / 256.0
    for i in range(256):
        r.freq.nu[i] = nu[i]
        r.csect[i].csect_HI, r.csect[i].csect_HeI, r.csect[i].csect_HeII = cs3[3 * i:3 * i + 3]
    return r


def _mesh_dev(fields):
    from argot_b200 import abi
    dens, fHI, fHeI, fHeII = fields
    m = np.zeros(len(dens), dtype=np.dtype(abi.FluidMesh))
    m["dens"] = dens
    m["chem"]["fHI"] = fHI
    m["chem"]["fHeI"] = fHeI
    m["chem"]["fHeII"] = fHeII
    m["prev_chem"]["GammaHI"] = 123.0  # must be overwritten by zero_out
    t = torch.from_numpy(m.view(np.uint8).copy()).cuda()
    return m, t


def _cuda(stream):
    from argot_b200 import abi
    cp = abi.CudaParam()
    cp.num_cuda_dev = 1
    cp.strm[0] = stream
    cm = (abi.CudaMemSpace * 1)()
    return cp, cm


@pytest.mark.parametrize("name", ["golden_march.npz", "golden_path_ragged.npz"])
def test_calc_optical_depth_cuda_bitwise(cuda_ok, name):
    from argot_b200 import _lib as L, abi
    lib = L.load()
    g = golden(name)
    edge = int(g["edge"])
    fields = tuple(g[k] for k in ("dens", "fHI", "fHeI", "fHeII"))
    _, mesh = _mesh_dev(fields)
    segs = g["seg"]
    seg = np.zeros(len(segs), dtype=np.dtype(abi.RaySegment))
    seg["ray_indx"] = np.arange(len(segs))
    for i, k in enumerate(("xpos_start", "ypos_start", "zpos_start", "xpos_end", "ypos_end", "zpos_end")):
        seg[k] = segs[:, i]
    seg["optical_depth_HI"] = -1.0
    run = _run_param(edge, float(g["lunit"]), float(g["denstonh"]), nseg=len(segs))
    cp, cm = _cuda(torch.cuda.current_stream().cuda_stream)
    cm[0].mesh_dev = mesh.data_ptr()
    lib.argot_b200_set_dropin_march_mode(0)
    lib.calc_optical_depth_cuda(seg.ctypes.data, C.addressof(cm), C.addressof(cp), C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    got = np.stack([seg["optical_depth_HI"], seg["optical_depth_HeI"], seg["optical_depth_HeII"]], 1)
    assert np.array_equal(got, g["tau"])
    # the positions and indices are left as they were
    assert np.array_equal(seg["xpos_end"], segs[:, 3])
    # Kahan mode: same call, FP64-closer columns
    lib.argot_b200_set_dropin_march_mode(1)
    lib.calc_optical_depth_cuda(seg.ctypes.data, C.addressof(cm), C.addressof(cp), C.addressof(run))
    lib.argot_b200_set_dropin_march_mode(0)
    got2 = np.stack([seg["optical_depth_HI"], seg["optical_depth_HeI"], seg["optical_depth_HeII"]], 1)
    ok = g["tau"] > 1e-6
    assert np.max(np.abs(got2 - g["tau"])[ok] / g["tau"][ok]) < 3e-4


@pytest.mark.parametrize("edge", [16, 19])
def test_dropin_rates_vs_reference(cuda_ok, edge):
    """zero_out_photoion_rate_cuda + calc_photoion_rate_cuda on the
    reference's own light rays, against the reference's calc_photoion_rate
    (19^3: a ragged mesh)."""
    from argot_b200 import _lib as L, abi, workload as W
    lib = L.load()
    wl = W.tiny(edge, 5, seed=77)
    R = ref_lib(edge)
    R.init(wl.lunit, wl.denstonh, 0.5, 1)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    R.zero_rates()
    out = R.run_range(0, edge ** 3, True, want=("tgt", "src", "tau", "spectra"))
    want = R.get_rates()
    nray = out["nray"]
    rays = np.zeros(nray, dtype=np.dtype(abi.LightRay))
    rays["src"]["xpos"] = out["src"][:, 0]
    rays["src"]["ypos"] = out["src"][:, 1]
    rays["src"]["zpos"] = out["src"][:, 2]
    rays["src"]["photon_rate"] = out["spectra"]
    rays["ix_target"], rays["iy_target"], rays["iz_target"] = out["tgt"].T
    rays["optical_depth_HI"], rays["optical_depth_HeI"], rays["optical_depth_HeII"] = out["tau"].T
    rays_io = np.zeros(nray, dtype=np.dtype(abi.LightRayIO))
    m, mesh = _mesh_dev(wl.fields())
    run = _run_param(edge, wl.lunit, wl.denstonh, nray=nray)
    cp, cm = _cuda(torch.cuda.current_stream().cuda_stream)
    cm[0].mesh_dev = mesh.data_ptr()
    lib.zero_out_photoion_rate_cuda(C.addressof(cm), C.addressof(cp), C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    lib.calc_photoion_rate_cuda(C.addressof(cm), rays.ctypes.data, rays_io.ctypes.data,
                                C.addressof(cp), C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    back = mesh.cpu().numpy().view(np.dtype(abi.FluidMesh))
    pc = back["prev_chem"]
    got = np.stack([pc["GammaHI"], pc["GammaHeI"], pc["GammaHeII"], pc["HeatHI"], pc["HeatHeI"],
                    pc["HeatHeII"]])
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < 2e-6, rel.max(axis=1)
    # the side effect the reference has: ray_IO filled from ray
    assert np.array_equal(rays_io["src"]["photon_rate"], out["spectra"])
    assert np.array_equal(rays_io["ix_target"], out["tgt"][:, 0])
    # calling again ADDS (the caller zeroes between passes)
    lib.calc_photoion_rate_cuda(C.addressof(cm), rays.ctypes.data, rays_io.ctypes.data,
                                C.addressof(cp), C.addressof(run))
    back2 = mesh.cpu().numpy().view(np.dtype(abi.FluidMesh))["prev_chem"]["GammaHI"]
    assert np.allclose(back2, 2 * want[0], rtol=1e-6)


def test_legacy_calc_optical_depth_bitwise(cuda_ok):
    """the older name (libargot_b200_legacy.so) runs the same march"""
    import os
    from argot_b200 import _lib as L, abi
    from conftest import ROOT
    lib = L.load()
    legacy = C.CDLL(os.path.join(ROOT, "argot_b200", "libargot_b200_legacy.so"), mode=C.RTLD_LOCAL)
    g = golden("golden_march.npz")
    edge = int(g["edge"])
    _, mesh = _mesh_dev(tuple(g[k] for k in ("dens", "fHI", "fHeI", "fHeII")))
    segs = g["seg"]
    seg = np.zeros(len(segs), dtype=np.dtype(abi.RaySegment))
    seg["ray_indx"] = np.arange(len(segs))
    for i, k in enumerate(("xpos_start", "ypos_start", "zpos_start", "xpos_end", "ypos_end", "zpos_end")):
        seg[k] = segs[:, i]
    run = _run_param(edge, float(g["lunit"]), float(g["denstonh"]), nseg=len(segs))
    cp, cm = _cuda(torch.cuda.current_stream().cuda_stream)
    cm[0].mesh_dev = mesh.data_ptr()
    lib.argot_b200_set_dropin_march_mode(0)
    legacy.calc_optical_depth(C.c_void_p(seg.ctypes.data), C.c_void_p(C.addressof(cm)), C.c_void_p(C.addressof(cp)),
                              C.c_void_p(C.addressof(run)))
    assert lib.argot_b200_last_error() == 0
    got = np.stack([seg["optical_depth_HI"], seg["optical_depth_HeI"], seg["optical_depth_HeII"]], 1)
    assert np.array_equal(got, g["tau"])
