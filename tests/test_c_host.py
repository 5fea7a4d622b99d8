"""A C program (tests/c_host/device_path.c) drives the device fast path
through the C ABI alone -- fields, tree, ray counts and offsets, then one
argot_b200_run_group -- and its rates equal the Python driver's bit for
bit: the library needs no Python on its host side."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    cc = shutil.which(os.environ.get("CC", "gcc"))
    if cc is None or not os.path.isdir(os.path.join(CUDA_HOME, "include")):
        pytest.skip("no C compiler or CUDA headers")
    exe = str(tmp_path / "device_path")
    libdir = os.path.join(ROOT, "argot_b200")
    cmd = [cc, "-O2", "-std=c99", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA_HOME, "include"),
           os.path.join(ROOT, "tests", "c_host", "device_path.c"), "-o", exe, "-L" + libdir, "-l:libargot_b200.so",
           "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_c_host_program_compiles(tmp_path):
    """the C program builds against the header and the library (no GPU)"""
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_c_host_equals_python_driver(cuda_ok, tmp_path):
    from argot_b200 import _lib as L
    from argot_b200 import workload as W
    from argot_b200.pipeline import Problem
    exe = _build(tmp_path)
    wl = W.tiny(24, 10, seed=8)
    pb = Problem(wl, "cuda:0")
    import torch
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda:0")
    want = pb.run(L.PRECISION_KAHAN, L.RATE_EXACT_F32, crossings=cnt).view(6, -1).cpu().numpy()
    n = wl.ncell
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([wl.edge, wl.nsrc], np.int32).tofile(f)
        np.array([wl.theta], np.float32).tofile(f)
        np.array([wl.lunit, wl.denstonh], np.float64).tofile(f)
        np.stack([np.asarray(a, np.float32).ravel() for a in wl.fields()]).tofile(f)
        np.ascontiguousarray(wl.src_pos, np.float32).tofile(f)
        np.ascontiguousarray(pb.spectra, np.float64).tofile(f)
    pb.close()
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.uint8)
    rates = out[:6 * n * 4].view(np.float32).reshape(6, n)
    cross = int(out[6 * n * 4:].view(np.uint64)[0])
    assert np.array_equal(rates, want)
    assert cross == int(cnt.item())
