"""Parity at the benchmark configurations.

Config 1 (64^3 uniform mesh, 16 sources, opening angle 0.5) on the whole
mesh; config 2 (128^3 lognormal, 256 sources), config 4 (192^3, 1024
sources), config 5 (256^3 sigma_ln 1.2, 4096 clustered sources) and three
members of the config-3 batch (48 problems of uneven size) on seeded runs
of target cells, which the reference's own group loop computes on their
own (setup_light_ray_range, src/setup_light_ray_tree.c:397;
oracle/sampled.py).

Tolerances, as in the other GPU tests:
  reference-order march and ray lists   bit for bit against O1 (ARGOT's C)
  FP64 rates                            2e-6 relative against O1
  compensated (Kahan) columns           1e-5 relative against the FP64 march
  FP32 rates                            1e-4 relative against the FP64 oracle
  surrogate rates                       1e-3 relative against the FP64 oracle
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F64_RTOL = 2e-6
TAU_RTOL = 1e-5
F32_RTOL = 1e-4
SUR_RTOL = 1e-3

CONFIGS = {
    # name: (workload factory, runs, cells per run); runs None = whole mesh
    "config1_plain64": (lambda W: W.plain(seed=1), None, 0),
    "config2_precision128": (lambda W: W.precision(seed=2), 16, 16),
    "config4_learned192": (lambda W: W.learned(seed=4), 16, 16),
    "config5_largest256": (lambda W: W.largest(seed=5), 16, 16),
}


def check_config(wl, runs, seed=11):
    import torch
    from argot_b200 import _lib as L
    from argot_b200 import surrogate as S
    from argot_b200.pipeline import Problem
    from oracle.sampled import SampledParity, z_runs
    sp = SampledParity(wl, None if runs is None else z_runs(wl.edge, runs[0], runs[1], seed))
    ref, f64 = sp.reference(), sp.fp64()
    assert len(ref["tgt"]) > 0
    pb = Problem(wl)
    out = {"rays": len(ref["tgt"]), "cells": len(sp.all_cells())}
    # reference order: the reference's rays, its columns bit for bit, FP64 rates
    r64, rays = sp.device(pb, L.PRECISION_REFERENCE, L.RATE_EXACT_F64, want_rays=True)
    same_list, same_tau = sp.same_rays(rays)
    assert same_list, "ray lists differ from the reference's"
    assert same_tau, "reference-order columns differ from the reference's"
    out["f64_vs_O1"] = e = max(sp.rate_errors(r64, ref["rates"]).values())
    assert e < F64_RTOL, sp.rate_errors(r64, ref["rates"])
    # compensated march + FP32 rates against the FP64 oracle pipeline
    r32, rays = sp.device(pb, L.PRECISION_KAHAN, L.RATE_EXACT_F32, want_rays=True)
    out["tau_vs_f64"] = e = sp.column_error_vs_f64(rays)
    assert e < TAU_RTOL, e
    out["f32_vs_f64"] = e = max(sp.rate_errors(r32, f64["rates"]).values())
    assert e < F32_RTOL, sp.rate_errors(r32, f64["rates"])
    # surrogate + FP32 fallback against the FP64 oracle pipeline
    pb.set_blackbody()
    sur = S.Surrogate.from_file()
    try:
        rs, _ = sp.device(pb, L.PRECISION_KAHAN, surrogate=sur)
    finally:
        sur.close()
    out["surrogate_vs_f64"] = e = max(sp.rate_errors(rs, f64["rates"]).values())
    assert e < SUR_RTOL, sp.rate_errors(rs, f64["rates"])
    pb.close()
    torch.cuda.empty_cache()
    return out


@pytest.mark.parametrize("name", list(CONFIGS))
def test_config_parity(cuda_ok, name):
    from argot_b200 import workload as W
    make, nruns, length = CONFIGS[name]
    wl = make(W)
    out = check_config(wl, None if nruns is None else (nruns, length))
    print(name, out)


def test_config3_batch_members(cuda_ok):
    """The batch's members are bit-equal to their solo runs (test_gpu_batch);
    here three members of the 48-problem config (the smallest, a middle and
    the largest mesh) go through the batch launch and are held to the FP64
    oracle on sampled cells."""
    import torch
    from argot_b200 import workload as W
    from argot_b200.batch import Batch
    from oracle.sampled import SampledParity, z_runs
    wls = W.batched(48, seed=3)
    order = sorted(range(len(wls)), key=lambda i: (wls[i].edge, wls[i].nsrc))
    pick = [order[0], order[len(order) // 2], order[-1]]
    B = Batch([wls[i] for i in pick], "cuda:0")
    B.graph_launch()
    torch.cuda.synchronize()
    B.check_device_error()
    for k, i in enumerate(pick):
        wl = wls[i]
        sp = SampledParity(wl, z_runs(wl.edge, 8, 16, seed=100 + i))
        got = B.rates[k].view(6, -1)[:, torch.from_numpy(sp.all_cells()).cuda()].cpu().numpy()
        err = sp.rate_errors(got, sp.fp64()["rates"])
        assert max(err.values()) < F32_RTOL, (wl.name, err)
    B.close()
