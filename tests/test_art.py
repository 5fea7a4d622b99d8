"""ART diffuse radiation (src/diffuse_photon): the library's angle table and
step-function factors against ARGOT's own setup_diffuse_photon, bit for bit
(CPU); the device kernels and the calc_diffuse_photon_radiation drop-in
against ARGOT's own CPU calc_diffuse_photon_radiation built here (GPU).

The reference adds each ray's I (1 - e^-tau) into its cells in its thread
order; the device does the same sums with float atomics in arbitrary order
and evaluates e^-tau in FP32 where the reference uses double exp/expm1, so
the rates agree to a few float ulps per term, not bit for bit: the tests
hold them to 1e-4 relative (measured: see the assertion messages)."""
import ctypes as C

import numpy as np
import pytest

from conftest import ref_lib

UENETOK = 1.0e4   # uene = 1 <-> T ~ 1e4 K x wmol


def _fields(edge, seed):
    """8 planes: dens, fHI, fHII, fHeI, fHeII, fHeIII, felec, uene (a
    partly ionised lognormal-ish mesh with T in ~[2e3, 5e4] K)"""
    rng = np.random.default_rng(seed)
    n = edge ** 3
    dens = np.exp(rng.normal(0.0, 0.8, n))
    xh = np.clip(rng.beta(0.6, 0.6, n), 1e-4, 1 - 1e-4)
    yhe = rng.dirichlet([1.0, 1.0, 1.0], n)
    felec = xh + 0.0811258278 * (yhe[:, 1] + 2 * yhe[:, 2])
    uene = 10.0 ** rng.uniform(-0.6, 0.8, n)
    return np.stack([dens, 1 - xh, xh, yhe[:, 0], yhe[:, 1], yhe[:, 2], felec, uene]).astype(np.float32)


def _ref(edge):
    R = ref_lib(edge)
    from argot_b200.workload import units
    lunit, denstonh = units()
    R.init(lunit, denstonh, 0.5, 1)
    R.art_init(UENETOK)
    return R, lunit, denstonh


def test_angle_table_and_step_factors_equal_reference():
    from argot_b200 import diffuse as D
    R, _, _ = _ref(16)
    d, bc, c8, st = R.art_table()
    d2, bc2, c82 = D.angle_table(D.NSIDE)
    assert len(d) == 12 * D.NSIDE ** 2
    assert np.array_equal(d, d2) and np.array_equal(bc, bc2) and np.array_equal(c8, c82)
    assert np.array_equal(st, D.step_factors())


def test_angle_table_properties():
    from argot_b200 import diffuse as D
    for nside in (1, 2, 4):
        d, bc, c8 = D.angle_table(nside)
        assert len(d) == 12 * nside ** 2 and c8.sum() == len(d)
        assert np.allclose(np.linalg.norm(d.astype(np.float64), axis=1), 1.0, atol=1e-6)
        # the start face is on the side the dominant component enters from
        face_axis = np.array([2, 2, 0, 0, 1, 1])[bc[:, 0]]
        assert np.all(np.abs(d[np.arange(len(d)), face_axis]) >= np.abs(d).max(axis=1) - 1e-6)
        # processing order: octant, then start face
        key = bc[:, 1] * 8 + bc[:, 0]
        assert np.all(np.diff(key) >= 0)
        # the directions cover the sphere evenly: the mean is ~0
        assert np.abs(d.mean(axis=0)).max() < 1e-6


def test_art_rejects_bad_arguments():
    from argot_b200 import _lib as L
    lib = L.load()
    buf = np.zeros(64, np.float32)
    ibuf = np.zeros(64, np.int32)
    assert lib.argot_b200_art_angle_table(0, buf.ctypes.data, ibuf.ctypes.data, None) == L.EINVAL
    h = C.c_void_p()
    bad = np.array([[0.5, 0.5, 0.7]], np.float32)
    bc = np.array([[6, 0]], np.int32)
    st = np.zeros(6, np.float32)
    assert lib.argot_b200_art_create(bad.ctypes.data, bc.ctypes.data, 1, st.ctypes.data, C.byref(h)) == L.EINVAL
    from argot_b200.pipeline import unit_box_grid
    g = unit_box_grid(8, 1.0, 1.0)
    assert lib.argot_b200_art_rates(None, C.byref(g), 1.0, None, None, None, 1, None, None) == L.EINVAL
    lib.calc_diffuse_photon_radiation(None, None, None, None, None, None, None)
    assert lib.argot_b200_last_error() == L.EINVAL


def _device_rates(edge, planes, lunit, denstonh, apass=None):
    import torch
    from argot_b200 import diffuse as D
    from argot_b200.pipeline import unit_box_grid
    g = unit_box_grid(edge, lunit, denstonh)
    f = torch.from_numpy(planes).cuda()
    r = torch.zeros(6 * edge ** 3, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    art = D.Diffuse()
    art.rates(g, UENETOK, f, r, angles_per_pass=apass, crossings=cnt)
    torch.cuda.synchronize()
    from argot_b200 import _lib as L
    L.check(L.load().argot_b200_check_device_error(torch.cuda.current_stream().cuda_stream), "device error")
    art.close()
    return r.view(6, -1).cpu().numpy(), int(cnt.item())


def _rel(got, want):
    got, want = got.astype(np.float64), want.astype(np.float64)
    scale = np.abs(want).max(axis=1, keepdims=True)
    big = np.abs(want) > 1e-6 * scale
    return (np.abs(got - want)[big] / np.abs(want)[big]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("edge", [16, 24, 32])
def test_art_rates_match_reference(cuda_ok, edge):
    R, lunit, denstonh = _ref(edge)
    planes = _fields(edge, 7 * edge)
    R.art_set_mesh(planes)
    want, _ = R.art_run()
    assert np.isfinite(want).all()
    got, steps = _device_rates(edge, planes, lunit, denstonh)
    assert np.isfinite(got).all()
    err = _rel(got, want)
    assert err < 1e-4, err
    # every direction sends edge^2 rays through the box: at least edge^3
    # ray-cell steps per direction
    assert steps >= 768 * edge ** 3
    # the batch size of angles does not change the result beyond the order
    # of the atomic sums
    got1, steps1 = _device_rates(edge, planes, lunit, denstonh, apass=1)
    assert steps1 == steps
    assert _rel(got1, got) < 1e-5


@pytest.mark.gpu
def test_art_dropin_through_mesh_dev(cuda_ok):
    """calc_diffuse_photon_radiation with the reference's GPU signature: the
    caller's angle table (here the reference's own) and mesh_dev; the
    rates are added to prev_chem, nothing else changes."""
    import torch
    from argot_b200 import _lib as L, abi
    edge = 16
    R, lunit, denstonh = _ref(edge)
    d, bc, c8, st = R.art_table()
    planes = _fields(edge, 99)
    R.art_set_mesh(planes)
    want, _ = R.art_run()
    n = edge ** 3
    m = np.zeros(n, dtype=np.dtype(abi.FluidMesh))
    m["dens"] = planes[0]
    for k, f in enumerate(("fHI", "fHII", "fHeI", "fHeII", "fHeIII", "felec")):
        m["prev_chem"][f] = planes[1 + k]
    m["prev_uene"] = planes[7]
    m["eneg"] = 5.0
    before = m.copy()
    dev = torch.from_numpy(m.view(np.uint8).copy()).cuda()

    class Angle(C.Structure):
        _fields_ = [("xovr", C.c_float), ("yovr", C.c_float), ("zovr", C.c_float),
                    ("base_id", C.c_short), ("corner_id", C.c_short)]

    class Step(C.Structure):
        _fields_ = [("HI", C.c_float * 2), ("HeI", C.c_float * 2), ("HeII", C.c_float * 2)]

    class HostDiffuse(C.Structure):
        _fields_ = [("corner_id_num", C.c_int * 8), ("step_fact", C.POINTER(Step)),
                    ("angle", C.POINTER(Angle))]

    angles = (Angle * len(d))()
    for i in range(len(d)):
        angles[i] = Angle(*d[i].tolist(), int(bc[i, 0]), int(bc[i, 1]))
    step = Step((C.c_float * 2)(*st[0:2]), (C.c_float * 2)(*st[2:4]), (C.c_float * 2)(*st[4:6]))
    hd = HostDiffuse((C.c_int * 8)(*c8.tolist()), C.pointer(step), C.cast(angles, C.POINTER(Angle)))
    run = abi.RunParam()
    for a in ("x", "y", "z"):
        setattr(run, f"nmesh_{a}_local", edge)
        setattr(run, f"nmesh_{a}_total", edge)
        setattr(run, f"delta_{a}", float(np.float32(1.0) / np.float32(edge)))
        setattr(run, f"{a}max", 1.0)
        setattr(run, f"{a}max_local", 1.0)
    run.lunit, run.denstonh, run.uenetok = lunit, denstonh, UENETOK
    cp = abi.CudaParam()
    cp.num_cuda_dev = 1
    cp.strm[0] = torch.cuda.current_stream().cuda_stream
    cm = (abi.CudaMemSpace * 1)()
    cm[0].mesh_dev = dev.data_ptr()
    lib = L.load()
    lib.calc_diffuse_photon_radiation(None, C.addressof(run), C.addressof(cm), C.addressof(cp),
                                      C.addressof(hd), None, None)
    assert lib.argot_b200_last_error() == 0
    got = dev.cpu().numpy().view(np.dtype(abi.FluidMesh))
    names = ("GammaHI", "GammaHeI", "GammaHeII", "HeatHI", "HeatHeI", "HeatHeII")
    rates = np.stack([got["prev_chem"][k] for k in names])
    err = _rel(rates, want)
    assert err < 1e-4, err
    for f in ("dens", "eneg", "chem", "prev_uene"):
        assert np.array_equal(got[f], before[f])
    for f in ("fHI", "fHII", "fHeI", "fHeII", "fHeIII", "felec"):
        assert np.array_equal(got["prev_chem"][f], before["prev_chem"][f])
