"""GPU parity of the march (calc_optical_depth) and the ray generation.

Tolerances: the reference-order kernels are bit-exact against the reference.
The Kahan kernel is scored against the FP64 oracle at <= 1e-5 relative (the
exact-path tolerance for optical depth) on every per-species column
(ray_segment.optical_depth_HI/HeI/HeII) and on the optical depth
tau_nu = sum_s N_s sigma_s(nu) in every one of the 256 frequency bins."""
import numpy as np
import pytest

from conftest import golden, ref_lib

pytestmark = pytest.mark.gpu

KAHAN_RTOL = 1e-5


def tau_nu_error(cols, cols64):
    from oracle.oracle import Oracle
    _, cs, _ = Oracle().tables()
    a = np.asarray(cols, np.float64) @ cs.astype(np.float64).T
    b = np.asarray(cols64, np.float64) @ cs.astype(np.float64).T
    ok = b > 1e-12 * b.max()
    return (np.abs(a - b)[ok] / b[ok]).max()


def column_error(cols, cols64, floor=0.0):
    """Largest relative error of the per-species columns that exceed
    `floor` times the ray's largest column (every positive column by
    default)."""
    cols64 = np.asarray(cols64, np.float64)
    ok = cols64 > floor * cols64.max(axis=1, keepdims=True)
    return (np.abs(np.asarray(cols, np.float64) - cols64)[ok] / cols64[ok]).max()


def test_march_segments_reference_bitwise_golden(cuda_ok):
    from argot_b200 import _lib as L
    from gpu_util import march_segments
    g = golden("golden_march.npz")
    f = tuple(g[k] for k in ("dens", "fHI", "fHeI", "fHeII"))
    tau = march_segments(int(g["edge"]), f, g["seg"], L.PRECISION_REFERENCE)
    assert np.array_equal(tau, g["tau"])


def test_march_segments_kahan_vs_fp64(cuda_ok, oracle):
    from argot_b200 import _lib as L
    from gpu_util import march_segments
    from oracle.oracle import unit_box_grid
    g = golden("golden_march.npz")
    f = tuple(np.ascontiguousarray(g[k]) for k in ("dens", "fHI", "fHeI", "fHeII"))
    edge = int(g["edge"])
    tau = march_segments(edge, f, g["seg"], L.PRECISION_KAHAN).astype(np.float64)
    t64 = oracle.march_f64(unit_box_grid(edge, 1.0, 1.0), f, g["seg"])
    assert tau_nu_error(tau, t64) < KAHAN_RTOL
    assert column_error(tau, t64) < KAHAN_RTOL
    # and closer to FP64 than the reference's own FP32 march
    assert tau_nu_error(tau, t64) < tau_nu_error(g["tau"], t64)
    assert column_error(tau, t64) < column_error(g["tau"], t64)


@pytest.mark.parametrize("edge,nsrc,theta", [(16, 6, 0.5), (19, 7, 0.6), (32, 24, 0.5), (32, 40, 0.7)])
def test_ray_lists_match_reference_tree(cuda_ok, edge, nsrc, theta):
    """Device tree walk emits, per target cell, the reference's rays in the
    reference's order (setup_light_ray_to)."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem
    wl = W.tiny(edge, nsrc, seed=edge + nsrc)
    wl.theta = theta
    pb, emit, tgt, tau, _ = run_problem(wl, L.PRECISION_REFERENCE, L.RATE_EXACT_F32)
    R = ref_lib(edge)
    R.init(wl.lunit, wl.denstonh, theta, 4)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    out = R.run_range(0, edge ** 3, False, want=("tgt", "src", "tau"))
    assert len(emit) == out["nray"]
    pos4, _ = pb.emitters()
    cell = lambda t: (t[:, 0].astype(np.int64) * edge + t[:, 1]) * edge + t[:, 2]  # noqa: E731
    # stable sort both lists by cell: the order within a cell must agree
    mine = np.argsort(cell(tgt), kind="stable")
    ref = np.argsort(cell(out["tgt"]), kind="stable")
    assert np.array_equal(cell(tgt)[mine], cell(out["tgt"])[ref])
    assert np.array_equal(pos4[emit[mine], :3], out["src"][ref])
    # and the columns of the reference-order march are the reference's
    assert np.array_equal(tau[mine], out["tau"][ref])


def test_ragged_golden_device_path(cuda_ok):
    """The whole device path on the ragged 19^3 golden problem (no axis a
    multiple of the 2x4x4 target blocks): per cell, the reference's rays in
    the reference's order, its columns bit for bit, its rates within the
    FP64 kernel's tolerance."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem
    g = golden("golden_path_ragged.npz")
    edge = int(g["edge"])
    wl = W.tiny(edge, len(g["src_rate"]), seed=5)
    wl.theta = float(g["theta"])
    for k in ("dens", "fHI", "fHeI", "fHeII", "src_pos", "src_rate"):
        assert np.array_equal(getattr(wl, k), g[k]), k
    pb, emit, tgt, tau, rates = run_problem(wl, L.PRECISION_REFERENCE, L.RATE_EXACT_F64)
    assert len(emit) == len(g["tgt"])
    pos4, _ = pb.emitters()
    cell = lambda t: (t[:, 0].astype(np.int64) * edge + t[:, 1]) * edge + t[:, 2]  # noqa: E731
    mine = np.argsort(cell(tgt), kind="stable")
    ref = np.argsort(cell(g["tgt"]), kind="stable")
    assert np.array_equal(cell(tgt)[mine], cell(g["tgt"])[ref])
    assert np.array_equal(pos4[emit[mine], :3], g["src"][ref])
    assert np.array_equal(tau[mine], g["tau"][ref])
    # the device exp (<= 1 ulp in double) moves the float rates by a few ulps
    want = g["rates"].astype(np.float64)
    rel = np.abs(rates - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < 2e-6, rel.max(axis=1)


def test_march_rays_kahan_vs_fp64(cuda_ok, oracle):
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem, ray_segments
    from oracle.oracle import unit_box_grid
    wl = W.tiny(32, 20, seed=8, sigma_ln=1.2)
    pb, emit, tgt, tau, _ = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)
    segs = ray_segments(pb, emit, tgt)
    t64 = oracle.march_f64(unit_box_grid(32, wl.lunit, wl.denstonh), wl.fields(), segs)
    err = tau_nu_error(tau, t64)
    assert err < KAHAN_RTOL, err
    cerr = column_error(tau, t64)
    assert cerr < KAHAN_RTOL, cerr
    # the reference's FP32 order is visibly less accurate on the same rays
    t32 = oracle.march_f32ref(unit_box_grid(32, wl.lunit, wl.denstonh), wl.fields(), segs)
    assert tau_nu_error(t32, t64) > err
    assert column_error(t32, t64) > cerr


@pytest.mark.parametrize("seed", [8, 21])
def test_march_rays_end_test_equals_face_counts(cuda_ok, seed):
    """The device path's march ends a ray when its next face lies past the
    end point (the target cell's centre); the explicit-segment march counts
    the faces of each axis instead.  Both take the same faces in the same
    order, so the columns are equal bit for bit."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import march_segments, run_problem, ray_segments
    wl = W.tiny(32, 20, seed=seed, sigma_ln=1.2)
    pb, emit, tgt, tau, _ = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)
    segs = ray_segments(pb, emit, tgt)
    tau_seg = march_segments(32, wl.fields(), segs, L.PRECISION_KAHAN, wl.lunit, wl.denstonh)
    assert len(segs) > 10000
    assert np.array_equal(tau, tau_seg)


def test_grouped_rays_equal_single_pass(cuda_ok):
    """Memory-bounded groups of target blocks give the same columns."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem
    wl = W.tiny(32, 12, seed=3)
    _, e1, t1, tau1, r1 = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)
    pb, e2, t2, tau2, r2 = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32, max_group_rays=5000)
    assert len(pb.groups) > 3
    assert np.array_equal(e1, e2) and np.array_equal(t1, t2)
    assert np.array_equal(tau1, tau2)
    assert np.array_equal(r1, r2)


def test_offsets_that_do_not_match_the_buffers_are_flagged(cuda_ok):
    """Block offsets past the caller's ray count (march, rates) or short of
    a block's rays (emission) set the device error flag
    and the kernels skip what does not fit.  The buffers here hold the full
    ray count, so nothing outside them is touched even without the checks."""
    import ctypes as C
    import torch
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from argot_b200.pipeline import Problem, RayGroup
    wl = W.tiny(16, 4, seed=2)
    pb = Problem(wl)
    g = pb.groups[0]
    rays, tau = pb.alloc_group_buffers()
    rates = torch.zeros(6 * pb.ncell, dtype=torch.float32, device="cuda")
    pb.emit(g, rays)
    pb.march(g, rays, tau)
    pb.rates(g, rays, tau, rates)
    torch.cuda.synchronize()
    pb.check_device_error()
    short = RayGroup(g.b0, g.b1, g.base, g.nray - 1)
    for step in (lambda: pb.march(short, rays, tau), lambda: pb.rates(short, rays, tau, rates),
                 lambda: pb.rates(short, rays, tau, rates, L.RATE_EXACT_F64)):
        step()
        torch.cuda.synchronize()
        with pytest.raises(L.ArgotError):
            pb.check_device_error()
        pb.check_device_error()  # the flag was cleared
    # emission: block 0's range one ray short, the later ranges shifted
    off = pb.blk_off.clone()
    off[1:] -= 1
    assert int(pb.blk_count[0]) > 1
    keep = rays.clone()
    L.check(pb.lib.argot_b200_emit_rays(C.byref(pb.grid), pb._dtree, g.b0, g.b1, off.data_ptr(), g.base,
                                        rays.data_ptr(), pb.sp), "emit")
    torch.cuda.synchronize()
    with pytest.raises(L.ArgotError):
        pb.check_device_error()
    # the rays of block 0 that fit are the same, the later blocks moved by one
    n0 = int(pb.blk_count[0])
    assert torch.equal(rays[:n0 - 1], keep[:n0 - 1])
    assert torch.equal(rays[n0 - 1:g.nray - 1], keep[n0:g.nray])
    pb.close()


def test_stitch_segmented_sum(cuda_ok, oracle):
    import torch
    from argot_b200 import _lib as L
    lib = L.load()
    rng = np.random.default_rng(5)
    nray = 3000
    nseg_per = rng.integers(0, 5, nray)
    ray_indx = np.repeat(np.arange(nray, dtype=np.uint64), nseg_per)
    seg_tau = rng.random((len(ray_indx), 3)).astype(np.float32)
    ri = torch.from_numpy(ray_indx.view(np.int64)).cuda()
    st = torch.from_numpy(seg_tau).cuda()
    out = torch.full((nray, 3), 7.0, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    L.check(lib.argot_b200_stitch(len(ray_indx), ri.data_ptr(), st.data_ptr(), nray, out.data_ptr(), s),
            "stitch")
    got = out.cpu().numpy()
    want = np.zeros((nray, 3))
    np.add.at(want, ray_indx.astype(np.int64), seg_tau.astype(np.float64))
    assert np.allclose(got, want, rtol=2e-7, atol=0)
    # one segment per ray (the reference's single-rank case): exact copy
    one = np.arange(nray, dtype=np.uint64)
    t1 = rng.random((nray, 3)).astype(np.float32)
    one_d = torch.from_numpy(one.view(np.int64)).cuda()
    t1_d = torch.from_numpy(t1).cuda()
    L.check(lib.argot_b200_stitch(nray, one_d.data_ptr(), t1_d.data_ptr(), nray, out.data_ptr(), s),
            "stitch")
    assert np.array_equal(out.cpu().numpy(), oracle.accum(nray, one, t1))


def test_stitch_flags_ray_index_past_the_rays(cuda_ok):
    """A segment whose ray index is past the caller's ray count is skipped
    and reported through the device error flag; the other rays are summed."""
    import torch
    from argot_b200 import _lib as L
    lib = L.load()
    nray = 100
    ray_indx = np.concatenate([np.arange(nray, dtype=np.uint64), np.array([nray, nray + 7], np.uint64)])
    seg_tau = np.ones((len(ray_indx), 3), np.float32)
    ri = torch.from_numpy(ray_indx.view(np.int64)).cuda()
    st = torch.from_numpy(seg_tau).cuda()
    out = torch.zeros((nray + 8, 3), dtype=torch.float32, device="cuda")  # room past nray: nothing may land there
    s = torch.cuda.current_stream().cuda_stream
    L.check(lib.argot_b200_stitch(len(ray_indx), ri.data_ptr(), st.data_ptr(), nray, out.data_ptr(), s), "stitch")
    torch.cuda.synchronize()
    with pytest.raises(L.ArgotError):
        L.check(lib.argot_b200_check_device_error(s), "device error flag")
    L.check(lib.argot_b200_check_device_error(s), "device error flag")  # cleared
    got = out.cpu().numpy()
    assert np.array_equal(got[:nray], np.ones((nray, 3), np.float32))
    assert not got[nray:].any()
