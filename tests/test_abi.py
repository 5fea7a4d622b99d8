"""The C-ABI library: builds, loads without a GPU, exports every symbol the
header declares, and its struct layouts equal the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, ref_lib


def header_functions():
    text = open(os.path.join(ROOT, "include", "argot_b200.h")).read()
    return sorted(set(re.findall(r"ARGOT_B200_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from argot_b200 import _lib
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    # and the binding covers every declared function
    assert set(declared) == set(_lib.exported_symbols())


def test_struct_layouts_match(tmp_path):
    from argot_b200 import _lib, abi
    lib = _lib.load()
    mine = np.zeros(10, np.uint64)
    lib.argot_b200_struct_sizes(mine.ctypes.data)
    assert list(mine) == abi.sizes()
    assert list(mine) == [56, 2384, 2096, 2072, 156, 52, 5480, 12, 2072, 24]
    assert lib.argot_b200_abi_check(mine.ctypes.data, 10) == 0
    bad = mine.copy()
    bad[1] += 8
    assert lib.argot_b200_abi_check(bad.ctypes.data, 10) == _lib.EINVAL
    R = ref_lib(16)
    assert list(R.struct_sizes()) == abi.sizes()
    assert list(R.struct_offsets()) == abi.offsets()


def test_tables_and_spectra_match_oracle(oracle):
    from argot_b200 import pipeline
    nu, cs = pipeline.tables()
    onu, ocs, _ = oracle.tables()
    assert np.array_equal(nu, onu) and np.array_equal(cs, ocs)
    from argot_b200 import _lib
    lib = _lib.load()
    out = np.zeros(256)
    for T, tot in ((1.0e5, 3.0e49), (4.0e4, 1.0e51)):
        lib.argot_b200_photon_rate(0, T, tot, out.ctypes.data)
        assert np.array_equal(out, oracle.photon_rate(0, T, tot))


def test_tree_builds_on_host():
    """Tree construction is host code: runs without a GPU."""
    from argot_b200 import _lib, workload as W
    from argot_b200.pipeline import photon_counts, unit_box_grid
    lib = _lib.load()
    wl = W.tiny(16, 9, seed=4)
    g = unit_box_grid(16, wl.lunit, wl.denstonh)
    spec = W.photon_rates(photon_counts, wl.src_type, wl.src_param, wl.src_rate)
    t = C.c_void_p()
    assert lib.argot_b200_tree_build(C.byref(g), wl.nsrc, wl.src_pos.ctypes.data,
                                     spec.ctypes.data, 0.5, C.byref(t)) == 0
    nn = lib.argot_b200_tree_num_nodes(t)
    ne = lib.argot_b200_tree_num_emitters(t)
    assert ne == nn + wl.nsrc and nn >= wl.nsrc
    pos4 = np.zeros((ne, 4), np.float32)
    sp = np.zeros((ne, 256))
    assert lib.argot_b200_tree_emitters(t, pos4.ctypes.data, sp.ctypes.data) == 0
    # root spectrum = sum of all sources; source emitters carry their own
    assert np.allclose(sp[0], spec.sum(axis=0), rtol=1e-13)
    assert np.array_equal(sp[nn:], spec)
    assert np.array_equal(pos4[nn:, :3], wl.src_pos)
    lib.argot_b200_tree_free(t)


def test_invalid_arguments_rejected_without_gpu():
    from argot_b200 import _lib
    lib = _lib.load()
    assert lib.argot_b200_tree_build(None, 0, None, None, 0.5, None) == _lib.EINVAL
    nb = C.c_uint64()
    assert lib.argot_b200_num_blocks(None, C.byref(nb)) == _lib.EINVAL
    assert lib.argot_b200_last_error() == _lib.EINVAL


def test_batch_and_surrogate_reject_bad_arguments():
    """Argument checks of the batch and surrogate entry points run before any
    CUDA call, so they answer on a host without a GPU."""
    import ctypes as C
    from argot_b200 import _lib as L
    from argot_b200.pipeline import unit_box_grid
    lib = L.load()
    h = C.c_void_p()
    assert lib.argot_b200_batch_create(None, 0, C.byref(h)) == L.EINVAL
    probs = (L.BatchProblem * 1)()
    probs[0] = L.BatchProblem(unit_box_grid(8, 1.0, 1.0), None, None, None, None, None, None)
    assert lib.argot_b200_batch_create(probs, 1, C.byref(h)) == L.EINVAL   # no buffers
    assert lib.argot_b200_batch_configure(None, None) == L.EINVAL
    assert lib.argot_b200_batch_run(None, None, None) == L.EINVAL
    assert lib.argot_b200_batch_graph_launch(None, None) == L.EINVAL
    assert lib.argot_b200_batch_tune(None, 1, None, None, None) == L.EINVAL
    assert lib.argot_b200_batch_num_items(None) == -1
    assert lib.argot_b200_surrogate_workspace(10) == 7 * 4 * 10
    assert lib.argot_b200_surrogate_create(None, None, 5e-4, C.byref(h)) == L.EINVAL
    g = unit_box_grid(8, 1.0, 1.0)
    assert lib.argot_b200_photoion_rays_surrogate(C.byref(g), None, None, None, 0, 1, None, 0, None, 0, None,
                                                  None, None, None, None) == L.EINVAL


def test_dropin_failure_is_logged_to_proc_file(tmp_path):
    """A drop-in that fails records its status and writes one line to the
    caller's run->proc_file, the reference's log."""
    import ctypes as C
    import ctypes.util
    from argot_b200 import _lib as L, abi
    libc = C.CDLL(ctypes.util.find_library("c"))
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    log = tmp_path / "proc.log"
    fp = libc.fopen(str(log).encode(), b"w")
    assert fp
    run = abi.RunParam()
    run.proc_file = fp
    run.nmesh_x_local = run.nmesh_y_local = run.nmesh_z_local = 8
    cm = (abi.CudaMemSpace * 1)()   # no mesh on the device: invalid
    lib = L.load()
    lib.calc_optical_depth_cuda(None, C.addressof(cm), None, C.addressof(run))
    assert lib.argot_b200_last_error() == L.EINVAL
    libc.fclose(fp)
    text = log.read_text()
    assert "calc_optical_depth_cuda" in text and "(-1)" in text


def test_dropins_reject_bad_mesh_sizes():
    """Non-positive local mesh sizes or cell widths are rejected before
    anything reaches the device.  The mesh pointer is a placeholder that is
    never dereferenced, so this runs only where no GPU is present."""
    import ctypes as C
    import torch
    from argot_b200 import _lib as L, abi
    if torch.cuda.is_available():
        pytest.skip("host-only argument checks")
    lib = L.load()
    cm = (abi.CudaMemSpace * 1)()
    cm[0].mesh_dev = 0x1000
    for nx, d in ((-1, 0.125), (8, 0.0), (0, 0.125)):
        run = abi.RunParam()
        run.nmesh_x_local, run.nmesh_y_local, run.nmesh_z_local = nx, 8, 8
        run.delta_x = run.delta_y = run.delta_z = d
        lib.zero_out_photoion_rate_cuda(C.addressof(cm), None, C.addressof(run))
        assert lib.argot_b200_last_error() == (L.EINVAL if nx <= 0 else L.ECUDA), (nx, d)
        seg = np.zeros(1, dtype=np.dtype(abi.RaySegment))
        run.nseg = 1
        lib.calc_optical_depth_cuda(seg.ctypes.data, C.addressof(cm), None, C.addressof(run))
        assert lib.argot_b200_last_error() == L.EINVAL, (nx, d)
        lib.calc_photoion_rate_cuda(C.addressof(cm), None, None, None, C.addressof(run))
        assert lib.argot_b200_last_error() == L.EINVAL, (nx, d)


def test_legacy_names_forward_to_the_library():
    """libargot_b200_legacy.so exports ARGOT's older GPU entry-point names
    (calc_optical_depth, calc_photoion_rate) and forwards them: the status
    lands in the main library's argot_b200_last_error."""
    import ctypes as C
    from argot_b200 import _lib as L
    lib = L.load()
    legacy = C.CDLL(os.path.join(ROOT, "argot_b200", "libargot_b200_legacy.so"), mode=C.RTLD_LOCAL)
    for name in ("calc_optical_depth", "calc_photoion_rate"):
        assert hasattr(legacy, name)
    text = open(os.path.join(ROOT, "include", "argot_b200_legacy.h")).read()
    assert set(re.findall(r"ARGOT_B200_API\s+void\s+(\w+)\s*\(", text)) == {"calc_optical_depth",
                                                                          "calc_photoion_rate"}
    lib.argot_b200_set_dropin_march_mode(0)
    legacy.calc_optical_depth(None, None, None, None)
    assert lib.argot_b200_last_error() == L.EINVAL
    lib.argot_b200_set_dropin_march_mode(0)
    assert lib.argot_b200_last_error() == 0
    legacy.calc_photoion_rate(None, None, None, None, None)
    assert lib.argot_b200_last_error() == L.EINVAL


def test_run_group_rejects_bad_arguments():
    import ctypes as C
    from argot_b200 import _lib as L
    from argot_b200.pipeline import unit_box_grid
    lib = L.load()
    g = unit_box_grid(8, 1.0, 1.0)
    off = np.zeros(17, np.uint64)
    # no buffers
    assert lib.argot_b200_run_group(C.byref(g), None, None, 0, 1, None, off.ctypes.data, 0, None, None, 0, 1, 1,
                                    4, None, None, None) == L.EINVAL
    # parts out of range, emit not 0/1
    fake = C.c_void_p(16)
    for parts, emit in ((0, 0), (5000, 0), (4, 2)):
        assert lib.argot_b200_run_group(C.byref(g), fake, fake, 0, 1, fake, off.ctypes.data, 0, fake, fake, emit, 1,
                                        1, parts, fake, None, None) == L.EINVAL
