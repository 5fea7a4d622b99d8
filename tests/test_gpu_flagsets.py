"""The drop-in built for ARGOT's other flag sets against the reference's own
C compiled with the same flags, on a seeded 16^3 mesh:
  * calc_optical_depth_cuda: every column (HI, HeI, HeII, HM, H2I, H2II as the
    set has them) bit-identical to calc_optical_depth (reference-order
    march), and within the reference's own FP32 spread in the compensated
    mode;
  * calc_photoion_rate_cuda after zero_out_photoion_rate_cuda: every Gamma
    and Heat field within 2e-6 of calc_photoion_rate (FP64 both; the device
    exp / pow differ by an ulp), for the photon-conserving and the plain
    branch, with the scale factor, and with the H2 Lyman-Werner term;
  * smooth_photoion_rate: every rate field bit-identical to the reference's
    smoothing, on the device mesh and in the host copy."""
import ctypes as C

import numpy as np
import pytest
import torch

from flagset_util import EDGE, Case, variant_lib

pytestmark = pytest.mark.gpu

TAGS = ["h2_pc", "he_h2_pc", "he", "he_pc_cosmo", "hi"]


def _cuda(mesh_dev):
    from argot_b200 import abi
    cp = abi.CudaParam()
    cp.num_cuda_dev = 1
    cp.strm[0] = torch.cuda.current_stream().cuda_stream
    cm = (abi.CudaMemSpace * 1)()
    cm[0].mesh_dev = mesh_dev.data_ptr()
    return cp, cm


def _to_dev(a):
    return torch.from_numpy(a.view(np.uint8).copy()).cuda()


def _from_dev(t, dtype):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype)


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_march_bitwise(cuda_ok, tag):
    cs = Case(tag, seed=11)
    lib = variant_lib(tag)
    mesh = _to_dev(cs.mesh_init)
    cp, cm = _cuda(mesh)
    seg_ref = cs.seg.copy()
    run_ref = cs.run_bytes(nseg=len(seg_ref))
    C.memmove(cs.run_ptr, C.addressof(run_ref), C.sizeof(run_ref))
    cs.R.calc_optical_depth(seg_ref.ctypes.data, cs.mesh_ref.ctypes.data, cs.run_ptr)
    run = cs.run_bytes(nseg=len(seg_ref))
    got = cs.seg.copy()
    lib.argot_b200_set_dropin_march_mode(0)
    lib.calc_optical_depth_cuda(got.ctypes.data, C.addressof(cm), C.addressof(cp), C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    for c in cs.Lay.columns:
        k = "optical_depth_" + c
        assert np.array_equal(got[k], seg_ref[k]), c
        assert (seg_ref[k] > 0).mean() > 0.9, c
    # the compensated march: within the reference's own FP32 spread
    kah = cs.seg.copy()
    lib.argot_b200_set_dropin_march_mode(1)
    lib.calc_optical_depth_cuda(kah.ctypes.data, C.addressof(cm), C.addressof(cp), C.addressof(run))
    lib.argot_b200_set_dropin_march_mode(0)
    assert lib.argot_b200_last_error() == 0
    for c in cs.Lay.columns:
        k = "optical_depth_" + c
        rel = np.abs(kah[k].astype(np.float64) - seg_ref[k]) / np.maximum(np.abs(seg_ref[k]), 1e-30)
        assert rel.max() < 5e-4, (c, rel.max())


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_rates_match_reference(cuda_ok, tag):
    cs = Case(tag, seed=12)
    lib = variant_lib(tag)
    nray = len(cs.ray)
    # the reference: zero, then add every ray (one thread: ray order)
    run_ref = cs.run_bytes(nray=nray)
    C.memmove(cs.run_ptr, C.addressof(run_ref), C.sizeof(run_ref))
    for k in cs.Lay.rates:
        cs.mesh_ref["prev_chem"][k] = 7.0
    cs.R.zero_out_photoion_rate(cs.mesh_ref.ctypes.data, cs.run_ptr)
    ray_ref = cs.ray.copy()
    cs.R.calc_photoion_rate(cs.mesh_ref.ctypes.data, ray_ref.ctypes.data, cs.run_ptr)
    want = cs.rates_of(cs.mesh_ref).astype(np.float64)
    # the drop-in on the device mesh
    m0 = cs.mesh_init.copy()
    for k in cs.Lay.rates:
        m0["prev_chem"][k] = 7.0  # zero_out must clear every field
    mesh = _to_dev(m0)
    cp, cm = _cuda(mesh)
    run = cs.run_bytes(nray=nray)
    lib.zero_out_photoion_rate_cuda(C.addressof(cm), C.addressof(cp), C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    ray = cs.ray.copy()
    ray_io = np.zeros(nray, dtype=np.dtype(cs.Lay.LightRayIO))
    lib.calc_photoion_rate_cuda(C.addressof(cm), ray.ctypes.data, ray_io.ctypes.data, C.addressof(cp),
                                C.addressof(run))
    assert lib.argot_b200_last_error() == 0
    got = cs.rates_of(_from_dev(mesh, np.dtype(cs.Lay.FluidMesh))).astype(np.float64)
    # ray_IO carries the rays' targets and columns
    for c in cs.Lay.columns:
        assert np.array_equal(ray_io["optical_depth_" + c], cs.ray["optical_depth_" + c])
    assert np.array_equal(ray_io["ix_target"], cs.ray["ix_target"])
    for j, k in enumerate(cs.Lay.rates):
        w, g = want[:, j], got[:, j]
        assert np.isfinite(w).all() and np.isfinite(g).all(), k
        scale = np.abs(w).max()
        assert scale > 0, k
        live = np.abs(w) > 1e-12 * scale
        assert np.abs(g[~live]).max(initial=0.0) <= 1e-12 * scale, k
        rel = np.abs(g[live] - w[live]) / np.abs(w[live])
        assert rel.max() < 2e-6, (k, rel.max())


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_smoothing_bitwise(cuda_ok, tag):
    cs = Case(tag, seed=13, nseg=1, nray=1)
    lib = variant_lib(tag)
    rng = np.random.default_rng(5)
    m0 = cs.mesh_init.copy()
    for k in cs.Lay.rates:
        m0["prev_chem"][k] = np.exp(rng.normal(0, 2, cs.ncell)).astype(np.float32)
    cs.mesh_ref[:] = m0
    cs.R.refv_smooth()
    want = cs.rates_of(cs.mesh_ref)
    mesh = _to_dev(m0)
    cp, cm = _cuda(mesh)
    run = cs.run_bytes()
    host = m0.copy()
    lib.smooth_photoion_rate(host.ctypes.data, C.addressof(run), C.addressof(cm), C.addressof(cp), None)
    assert lib.argot_b200_last_error() == 0
    assert np.array_equal(cs.rates_of(_from_dev(mesh, np.dtype(cs.Lay.FluidMesh))), want)
    assert np.array_equal(cs.rates_of(host), want)
    assert not np.array_equal(want, cs.rates_of(m0))
