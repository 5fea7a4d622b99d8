"""Rate smoothing (smooth_photoion_rate.c): the CPU restatement in
oracle/smooth.py against ARGOT's own C built here, bit for bit, with the
reference Makefile's default isolated faces and with periodic faces; and the
CUDA stencil (argot_b200_smooth_rates) against both."""
import numpy as np
import pytest

from conftest import ref_lib
from oracle import smooth as SM


def _rates(edge, seed):
    rng = np.random.default_rng(seed)
    r = (10.0 ** rng.uniform(-16, -9, (6, edge ** 3))).astype(np.float32)
    r[:, rng.random(edge ** 3) < 0.05] = 0.0   # cells that received nothing
    r[3:] *= np.float32(1e-11)                 # heating rates are ~1e-11 of the Gammas
    return r


def _ref(edge, isolated):
    from oracle.oracle import RefLib
    import os
    from oracle import build
    ref_lib(edge)  # skips when no reference build can be had
    path = build.ref_lib_path(edge, isolated=isolated)
    if not os.path.exists(path) and not build.reference_available():
        pytest.skip("reference build unavailable")
    R = RefLib(edge, isolated=isolated)
    R.init(1.0, 1.0, 0.5, 1)
    return R


@pytest.mark.parametrize("isolated", [True, False])
@pytest.mark.parametrize("edge", [16, 32])
def test_restatement_equals_reference(edge, isolated):
    R = _ref(edge, isolated)
    x = _rates(edge, edge + isolated)
    assert np.array_equal(SM.smooth_rates(x, edge, isolated), R.smooth_rates(x))


def test_uniform_field_is_fixed():
    x = np.full((6, 8 ** 3), 3.0e-12, np.float32)
    for iso in (True, False):
        y = SM.smooth_rates(x, 8, iso)
        assert np.allclose(y, x, rtol=1e-6)


def test_entry_point_rejects_bad_arguments():
    import ctypes as C
    from argot_b200 import _lib as L
    from argot_b200.pipeline import unit_box_grid
    lib = L.load()
    g = unit_box_grid(8, 1.0, 1.0)
    assert lib.argot_b200_smooth_rates(C.byref(g), None, None, 1, None) == L.EINVAL
    buf = np.zeros(6 * 8 ** 3, np.float32)
    p = buf.ctypes.data
    assert lib.argot_b200_smooth_rates(C.byref(g), p, p, 1, None) == L.EINVAL   # aliasing
    assert lib.argot_b200_smooth_rates(C.byref(g), p, p + 4, 2, None) == L.EINVAL  # mode


@pytest.mark.gpu
@pytest.mark.parametrize("isolated", [True, False])
@pytest.mark.parametrize("edge", [16, 24, 32])
def test_device_smoothing_bit_identical(cuda_ok, edge, isolated):
    import torch
    from argot_b200 import _lib as L
    from argot_b200.pipeline import unit_box_grid
    import ctypes as C
    lib = L.load()
    g = unit_box_grid(edge, 1.0, 1.0)
    x = _rates(edge, 3 * edge + isolated)
    xin = torch.from_numpy(x.ravel()).cuda()
    out = torch.full_like(xin, -1.0)
    L.check(lib.argot_b200_smooth_rates(C.byref(g), xin.data_ptr(), out.data_ptr(), int(isolated),
                                        torch.cuda.current_stream().cuda_stream), "smooth_rates")
    got = out.view(6, -1).cpu().numpy()
    assert np.array_equal(got, SM.smooth_rates(x, edge, isolated))
    if edge in (16, 32):
        assert np.array_equal(got, _ref(edge, isolated).smooth_rates(x))


def test_dropin_smoothing_rejects_bad_arguments():
    from argot_b200 import _lib as L
    lib = L.load()
    assert lib.argot_b200_set_dropin_smooth_faces(2) == L.EINVAL
    assert lib.argot_b200_set_dropin_smooth_faces(-1) == L.EINVAL
    lib.smooth_photoion_rate(None, None, None, None, None)
    assert lib.argot_b200_last_error() == L.EINVAL
    assert lib.argot_b200_set_dropin_smooth_faces(1) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("isolated", [True, False])
@pytest.mark.parametrize("edge", [16, 24])
def test_dropin_smooth_photoion_rate(cuda_ok, edge, isolated):
    """smooth_photoion_rate with the reference's GPU-build signature: the
    rates of mesh_dev smoothed in place on the device, bit-identical to the
    reference, the same values written to the host mesh, every other field
    left as it was."""
    import ctypes as C
    import torch
    from argot_b200 import _lib as L, abi
    lib = L.load()
    x = _rates(edge, 5 * edge + isolated)
    names = ("GammaHI", "GammaHeI", "GammaHeII", "HeatHI", "HeatHeI", "HeatHeII")
    rng = np.random.default_rng(edge)
    m = np.zeros(edge ** 3, dtype=np.dtype(abi.FluidMesh))
    m["dens"] = rng.uniform(0.5, 2.0, edge ** 3)
    m["chem"]["fHI"] = rng.uniform(0, 1, edge ** 3)
    m["chem"]["GammaHI"] = 7.0
    m["prev_uene"] = 3.0
    for k, n in enumerate(names):
        m["prev_chem"][n] = x[k]
    before = m.copy()
    dev = torch.from_numpy(m.view(np.uint8).copy()).cuda()
    run = abi.RunParam()
    for a in ("x", "y", "z"):
        setattr(run, f"nmesh_{a}_local", edge)
        setattr(run, f"nmesh_{a}_total", edge)
    cp = abi.CudaParam()
    cp.num_cuda_dev = 1
    cp.strm[0] = torch.cuda.current_stream().cuda_stream
    cm = (abi.CudaMemSpace * 1)()
    cm[0].mesh_dev = dev.data_ptr()
    faces = 1 if isolated else 0
    assert lib.argot_b200_set_dropin_smooth_faces(faces) == 0
    try:
        want = SM.smooth_rates(x, edge, isolated)
        host = m.copy()
        lib.smooth_photoion_rate(host.ctypes.data, C.addressof(run), C.addressof(cm), C.addressof(cp), None)
        assert lib.argot_b200_last_error() == 0
        got_dev = dev.cpu().numpy().view(np.dtype(abi.FluidMesh))
        for k, n in enumerate(names):
            assert np.array_equal(got_dev["prev_chem"][n], want[k]), n
            assert np.array_equal(host["prev_chem"][n], want[k]), n
        # nothing else changes, on the device or on the host
        for arr in (got_dev, host):
            for f in ("dens", "chem", "prev_uene"):
                assert np.array_equal(arr[f], before[f])
            for f in ("wmol", "felec", "fHI", "fHII", "fHeI", "fHeII", "fHeIII"):
                assert np.array_equal(arr["prev_chem"][f], before["prev_chem"][f])
        if edge == 16:
            assert np.array_equal(want, _ref(edge, isolated).smooth_rates(x))
        # without a host mesh only the device copy changes (a second pass)
        lib.smooth_photoion_rate(None, C.addressof(run), C.addressof(cm), C.addressof(cp), None)
        assert lib.argot_b200_last_error() == 0
        twice = SM.smooth_rates(want, edge, isolated)
        got2 = dev.cpu().numpy().view(np.dtype(abi.FluidMesh))
        for k, n in enumerate(names):
            assert np.array_equal(got2["prev_chem"][n], twice[k]), n
    finally:
        lib.argot_b200_set_dropin_smooth_faces(1)
