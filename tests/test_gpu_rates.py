"""GPU parity of the photo-ionisation / heating rates (calc_photoion_rate).

EXACT_F64 follows the reference's FP64 algorithm and float accumulation
order; its only difference from the CPU is the device `exp` (<= 1 ulp in
double), so per-cell rates agree with the reference to a few float ulps:
tolerance 2e-6 relative.  EXACT_F32 (FP32, FP64 only in the small-dtau
photon-conserving factor) is scored against the FP64 oracle pipeline
(FP64 march + FP64 rates): tolerance 1e-4 relative."""
import numpy as np
import pytest

from conftest import ref_lib

pytestmark = pytest.mark.gpu

F64_RTOL = 2e-6
F32_RTOL = 1e-4


def _ref_spectra(pb, emit):
    _, spec = pb.emitters()
    return spec[emit]


def test_exact_f64_matches_oracle_on_device_rays(cuda_ok, oracle):
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem, ray_segments
    from oracle.oracle import unit_box_grid
    wl = W.tiny(32, 16, seed=21)
    pb, emit, tgt, tau, rates = run_problem(wl, L.PRECISION_REFERENCE, L.RATE_EXACT_F64)
    grid = unit_box_grid(32, wl.lunit, wl.denstonh)
    segs = ray_segments(pb, emit, tgt)
    want = oracle.photoion_f64ref(grid, wl.fields(), tau, tgt, segs[:, :3], _ref_spectra(pb, emit))
    rel = np.abs(rates - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < F64_RTOL, rel.max(axis=1)


@pytest.mark.parametrize("edge,nsrc,seed", [(32, 24, 31), (19, 9, 37)])
def test_exact_f64_end_to_end_vs_reference_build(cuda_ok, edge, nsrc, seed):
    """Whole path on the device (tree walk, reference-order march, FP64
    rates) against ARGOT's own C on the same seeded problem; 19^3 is a
    ragged mesh (no axis a multiple of the 2x4x4 target blocks)."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem
    wl = W.tiny(edge, nsrc, seed=seed)
    _, _, _, _, rates = run_problem(wl, L.PRECISION_REFERENCE, L.RATE_EXACT_F64)
    R = ref_lib(edge)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    R.zero_rates()
    R.run_range(0, edge ** 3, True, want=())
    want = R.get_rates()
    rel = np.abs(rates - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < F64_RTOL, rel.max(axis=1)


@pytest.mark.parametrize("edge", [32, 19])
def test_exact_f32_vs_fp64_oracle(cuda_ok, oracle, edge):
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem, ray_segments
    from oracle.oracle import unit_box_grid
    wl = W.tiny(edge, 16, seed=41, sigma_ln=1.2)
    pb, emit, tgt, tau, rates = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)
    grid = unit_box_grid(edge, wl.lunit, wl.denstonh)
    segs = ray_segments(pb, emit, tgt)
    t64 = oracle.march_f64(grid, wl.fields(), segs)
    want = oracle.photoion_f64(grid, wl.fields(), t64, tgt, segs[:, :3], _ref_spectra(pb, emit))
    rel = np.abs(rates.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < F32_RTOL, rel.max(axis=1)


def test_rates_deterministic(cuda_ok):
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from gpu_util import run_problem
    wl = W.tiny(32, 10, seed=2)
    a = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)[4]
    b = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F32)[4]
    assert np.array_equal(a, b)


def test_single_source_vacuum_known_answer(cuda_ok):
    """Known answer: one source in an optically thin uniform medium; the
    photon-conserving rate tends to the non-PC flux integral
    sum_nu Ndot_nu sigma_nu / (4 pi r^2 lunit^2) as dtau -> 0."""
    from argot_b200 import workload as W
    from argot_b200 import _lib as L
    from argot_b200.pipeline import photon_counts, tables
    from gpu_util import run_problem
    wl = W.plain(16, 1, seed=5)
    wl.dens[:] = 1.0e-6
    wl.src_pos[:] = np.float32(0.5 / 16 + 8 / 16)
    rates = run_problem(wl, L.PRECISION_KAHAN, L.RATE_EXACT_F64)[4]
    nu, cs = tables()
    spec = W.photon_rates(photon_counts, wl.src_type, wl.src_param, wl.src_rate)[0]
    d = 1.0 / 16
    ix = np.array([3, 8, 8])  # 5 cells from the source along -x
    c = (ix + 0.5) * d
    r = np.linalg.norm(c - wl.src_pos[0].astype(np.float64)) * wl.lunit
    fluxint = np.sum(spec * cs[:, 0]) / (4 * np.pi * r * r)
    got = rates[0, (ix[0] * 16 + ix[1]) * 16 + ix[2]]
    # thin shell vs point flux: (r^2 delta)/(r^2 delta + delta^3/12)
    assert abs(got / fluxint - 1.0) < 5e-3


def test_overlapped_run_equals_sequential(cuda_ok):
    """Problem.run(overlap=P): the march of one part on one stream while the
    rates of the previous part run on another gives the same field bit for
    bit, with the rays emitted inside the run or kept from before."""
    import torch
    from argot_b200 import _lib as L
    from argot_b200 import workload as W
    from argot_b200.pipeline import Problem
    wl = W.tiny(32, 16, seed=61, sigma_ln=1.2)
    pb = Problem(wl)
    bufs = pb.alloc_group_buffers()
    want = pb.run(L.PRECISION_KAHAN, L.RATE_EXACT_F32, buffers=bufs).clone()
    for parts in (2, 5, 8):
        got = pb.run(L.PRECISION_KAHAN, L.RATE_EXACT_F32, buffers=bufs, overlap=parts)
        torch.cuda.synchronize()
        assert torch.equal(got, want), parts
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    got = pb.run(L.PRECISION_KAHAN, L.RATE_EXACT_F32, buffers=bufs, crossings=cnt, keep_rays=True, overlap=3)
    torch.cuda.synchronize()
    assert torch.equal(got, want) and int(cnt.item()) > 0
    pb.check_device_error()
