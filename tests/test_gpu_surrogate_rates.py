"""The surrogate rate path (BF16 network on the tensor cores, exact FP32
fallback) against the FP64 oracle pipeline (FP64 march + FP64 rates of
calc_photoion_rate.c:159-425): per-cell Gamma and heating within 1e-3
relative.  The network's gain is the share of rays it serves within each
cell's error budget; an untrained network, with the envelope of its own
errors, serves far fewer."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUR_RTOL = 1e-3


def _weights():
    from argot_b200 import surrogate as S
    if not os.path.exists(S.WEIGHTS):
        pytest.fail(f"trained weights missing: {S.WEIGHTS} (python -m argot_b200.train_surrogate)")
    return S.Surrogate.from_file()


def _run(wl, sur):
    import torch
    from argot_b200 import _lib as L
    from argot_b200.pipeline import Problem
    pb = Problem(wl)
    pb.set_blackbody()
    rays, tau = pb.alloc_group_buffers()
    rates = torch.zeros(6 * pb.ncell, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    emit, tgt = [], []
    for g in pb.groups:
        pb.emit(g, rays)
        pb.march(g, rays, tau, L.PRECISION_KAHAN)
        pb.rates_surrogate(g, rays, tau, rates, sur, cnt)
        e, t, _ = pb.ray_table(rays, g)
        emit.append(e)
        tgt.append(t)
    torch.cuda.synchronize()
    pb.check_device_error()
    return (pb, np.concatenate(emit), np.concatenate(tgt), rates.view(6, -1).cpu().numpy(),
            cnt.cpu().numpy())


def _fp64_oracle(oracle, pb, emit, tgt):
    from gpu_util import ray_segments
    from oracle.oracle import unit_box_grid
    wl = pb.wl
    grid = unit_box_grid(wl.edge, wl.lunit, wl.denstonh)
    segs = ray_segments(pb, emit, tgt)
    t64 = oracle.march_f64(grid, wl.fields(), segs)
    _, spec = pb.emitters()
    return oracle.photoion_f64(grid, wl.fields(), t64, tgt, segs[:, :3], spec[emit])


def _rel(got, want):
    return np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-300)


def test_surrogate_rates_neutral_vs_fp64_oracle(cuda_ok, oracle):
    """A mostly neutral mesh: most rays are optically thick at the edges,
    where the network's relative error |y| dq is large, so most of them
    fall back; the field stays within 1e-3."""
    from argot_b200 import workload as W
    sur = _weights()
    wl = W.tiny(32, 16, seed=41, sigma_ln=1.2)
    pb, emit, tgt, rates, cnt = _run(wl, sur)
    want = _fp64_oracle(oracle, pb, emit, tgt)
    rel = _rel(rates, want)
    print(f"neutral: surrogate served {cnt[0] / cnt.sum():.3f} of {cnt.sum()} rays; max rel {rel.max(axis=1)}")
    assert rel.max() < SUR_RTOL, rel.max(axis=1)
    assert cnt.sum() == len(emit)


@pytest.mark.parametrize("edge", [32, 19])
def test_surrogate_rates_ionized_vs_fp64_oracle(cuda_ok, oracle, edge):
    """An ionised mesh (thin rays): the network serves most rays and the
    field stays within 1e-3 of the FP64 oracle (19^3: a ragged mesh, no
    axis a multiple of the 2x4x4 target blocks)."""
    from argot_b200 import workload as W
    sur = _weights()
    wl = W.ionized(edge, 16, seed=42)
    pb, emit, tgt, rates, cnt = _run(wl, sur)
    want = _fp64_oracle(oracle, pb, emit, tgt)
    rel = _rel(rates, want)
    served = cnt[0] / cnt.sum()
    print(f"ionized: surrogate served {served:.3f} of {cnt.sum()} rays; max rel {rel.max(axis=1)}")
    assert rel.max() < SUR_RTOL, rel.max(axis=1)
    assert cnt.sum() == len(emit)
    assert served > 0.5  # rays that skip the 256-bin loop


def test_mixed_spectra_fall_back(cuda_ok, oracle):
    """Power-law sources (and tree nodes that merge them) are not single
    blackbodies: their rays take the exact quadrature, still within 1e-3."""
    from argot_b200 import workload as W
    sur = _weights()
    wl = W.tiny(32, 16, seed=43, sigma_ln=1.0)
    wl.src_type = wl.src_type.copy()
    wl.src_param = wl.src_param.copy()
    wl.src_type[::2] = 1
    wl.src_param[::2] = 1.5
    pb, emit, tgt, rates, cnt = _run(wl, sur)
    want = _fp64_oracle(oracle, pb, emit, tgt)
    assert _rel(rates, want).max() < SUR_RTOL
    assert cnt[1] > 0 and cnt.sum() == len(emit)


def test_trained_network_gain(cuda_ok, oracle):
    """What the trained network gains over the method without it: with the
    envelope of its own validated errors an untrained network keeps the
    same accuracy but serves far fewer rays (the rest fall back to the
    256-bin quadrature), while the trained one serves most of them (on an
    ionised mesh, where the rays are thin enough for the network)."""
    from argot_b200 import surrogate as S
    from argot_b200 import workload as W
    trained = _weights()
    tr = S.Trainer("cuda", nT=64, seed=5)
    Xv, Yv = tr.samples(200_000, seed=77)
    untrained = S.Surrogate(S.init_params(0), np.zeros((6, S.ENV_BINS), np.float32), tol=1.0)
    env = S.error_envelope(untrained.eval(Xv).cpu().numpy(), Yv.cpu().numpy())
    untrained = S.Surrogate(S.init_params(0), env, tol=5e-4)
    wl = W.ionized(32, 16, seed=42)
    served = {}
    for name, sur in (("trained", trained), ("untrained", untrained)):
        pb, emit, tgt, rates, cnt = _run(wl, sur)
        want = _fp64_oracle(oracle, pb, emit, tgt)
        assert _rel(rates, want).max() < SUR_RTOL, name
        served[name] = cnt[0] / cnt.sum()
    print("served fraction", served)
    assert served["trained"] > served["untrained"] + 0.3


def test_surrogate_rates_deterministic(cuda_ok):
    from argot_b200 import workload as W
    sur = _weights()
    wl = W.tiny(32, 8, seed=44)
    a = _run(wl, sur)[3]
    b = _run(wl, sur)[3]
    assert np.array_equal(a, b)
