"""ARGOT's own GPU entry points (calc_optical_depth_cuda,
calc_photoion_rate_cuda, zero_out_photoion_rate_cuda), compiled for sm_100a
with the reference's nvcc flags by oracle/build.py, on the golden 16^3
problem: they are the reference-GPU baseline of bench.py, so they must
compute the path's results.  The reference's GPU build is not bit-identical
to its CPU build (it compiles with -use_fast_math and contracts to FMA, and
sums the per-cell rates with float atomics in arbitrary order); the bounds
below are that spread, measured, not a property of this repository's
kernels, which match the CPU build bit for bit."""
import os

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _refgpu(g):
    from oracle import build
    from oracle.oracle import RefGpu
    edge = int(g["edge"])
    if not os.path.exists(build.refgpu_lib_path(edge)) and not build.reference_available():
        pytest.skip("reference GPU build unavailable")
    R = RefGpu(edge)
    R.init(float(g["lunit"]), float(g["denstonh"]), float(g["theta"]), 4)
    R.set_mesh(g["dens"], g["fHI"], g["fHeI"], g["fHeII"])
    R.set_sources(g["src_type"], g["src_param"], g["src_pos"], g["src_rate"])
    R.upload()
    return R, edge


def test_reference_gpu_path_computes_the_path(cuda_ok):
    g = golden("golden_path.npz")
    R, edge = _refgpu(g)
    try:
        R.zero_rates_gpu()
        out = R.run_range_gpu(0, edge ** 3, kernel_reps=1, want=("seg", "tau"))
        assert out["nray"] == len(g["tgt"]) and out["nseg"] == len(g["tgt"])
        # the reference's own tree builds the same segments on the host
        assert np.array_equal(out["seg"], g["seg"])
        # columns: the fast-math GPU march against the CPU build
        tau, ref = out["tau"].astype(np.float64), g["tau"].astype(np.float64)
        big = ref > 1e-6 * ref.max(axis=1, keepdims=True)
        rel = np.abs(tau - ref)[big] / ref[big]
        assert rel.max() < 1e-4, rel.max()
        # per-cell rates
        rates = R.rates_gpu().astype(np.float64)
        want = g["rates"].astype(np.float64)
        nz = want > 0
        assert np.array_equal(rates > 0, nz)
        rrel = np.abs(rates - want)[nz] / want[nz]
        assert rrel.max() < 1e-3, rrel.max()
        # the kernel-only passes ran and took time
        assert out["march_kernel_ms"] > 0 and out["rate_kernel_ms"] > 0
    finally:
        R.close()


def test_reference_loop_with_this_librarys_entry_points(cuda_ok):
    """ARGOT's group loop (its tree, its host light rays, its accum) with
    libargot_b200's calc_optical_depth_cuda / calc_photoion_rate_cuda linked
    in: columns bit for bit those of the reference's CPU build, rates within
    the device exp's few ulps."""
    from argot_b200 import _lib as L
    g = golden("golden_path.npz")
    R, edge = _refgpu(g)
    try:
        R.use_entry_points(L.load())
        R.zero_rates_gpu()
        out = R.run_range_gpu(0, edge ** 3, want=("seg", "tau"))
        assert np.array_equal(out["tau"], g["tau"])
        rates = R.rates_gpu().astype(np.float64)
        want = g["rates"].astype(np.float64)
        nz = want > 0
        assert np.array_equal(rates > 0, nz)
        assert (np.abs(rates - want)[nz] / want[nz]).max() < 2e-6
    finally:
        R.use_entry_points(None)
        R.close()
