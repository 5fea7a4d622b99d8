"""ARGOT's on-disk formats (argot_b200/formats.py) against the reference's
own writers and readers (output_data.c, input_data.c) built here: files the
reference writes read back field for field, files written here read by the
reference, and (on the GPU) the path run on a mesh and sources loaded from
reference-written files equal to the reference's own run on them."""
import ctypes as C
import os

import numpy as np
import pytest

from argot_b200 import abi
from argot_b200 import formats as F
from conftest import ref_lib


def _loaded_ref(wl):
    R = ref_lib(wl.edge)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    return R


def test_struct_sizes():
    assert C.sizeof(abi.FluidMeshIO) == 80
    assert F.SRC_DTYPE.itemsize == C.sizeof(abi.RadiationSrc) == 2072
    assert F.MESH_DTYPE.itemsize == 80


def test_reference_files_read_here(tmp_path):
    from argot_b200 import workload as W
    wl = W.tiny(16, 6, seed=7)
    R = _loaded_ref(wl)
    mesh, prefix = str(tmp_path / "run_000_000_000"), str(tmp_path / "run")
    R.write_files(mesh, prefix)
    hdr, cells = F.read_mesh(mesh)
    assert (hdr.nmesh_x_local, hdr.nmesh_x_total, hdr.mpi_nproc) == (16, 16, 1)
    assert hdr.lunit == wl.lunit and hdr.denstonh == wl.denstonh
    assert np.array_equal(cells["dens"], wl.dens)
    assert np.array_equal(cells["chem"]["fHI"], wl.fHI)
    assert np.array_equal(cells["chem"]["fHeI"], wl.fHeI)
    assert np.array_equal(cells["chem"]["fHeII"], wl.fHeII)
    freq, src = F.read_src(prefix + "_src.dat")
    assert len(src) == wl.nsrc
    assert np.array_equal(src["type"], wl.src_type)
    assert np.array_equal(np.stack([src["xpos"], src["ypos"], src["zpos"]], 1), wl.src_pos)
    assert np.array_equal(src["photon_rate"], R.source_spectra())
    assert freq == bytes(F.default_freq_param())
    back = F.workload_from_files(mesh, prefix + "_src.dat")
    assert np.array_equal(back.fHeII, wl.fHeII) and np.array_equal(back.src_spectra, R.source_spectra())


def test_files_written_here_read_by_reference(tmp_path):
    from argot_b200 import workload as W
    wl = W.tiny(16, 5, seed=9)
    R = _loaded_ref(wl)
    spec = R.source_spectra()
    mesh, srcf = str(tmp_path / "mine_000_000_000"), str(tmp_path / "mine_src.dat")
    F.write_mesh(mesh, F.mesh_header(16, wl.lunit, wl.denstonh), *wl.fields())
    F.write_src(srcf, wl.src_type, wl.src_param, wl.src_pos, spec)
    (dens, fHI, fHeI, fHeII), (typ, par, xyz, sp) = R.read_files(mesh, srcf)
    for a, b in zip((dens, fHI, fHeI, fHeII), wl.fields()):
        assert np.array_equal(a, b)
    assert np.array_equal(typ, wl.src_type) and np.array_equal(par, wl.src_param)
    assert np.array_equal(xyz, wl.src_pos) and np.array_equal(sp, spec)


def test_truncated_files_are_rejected(tmp_path):
    p = tmp_path / "short_src.dat"
    p.write_bytes(np.uint64(3).tobytes() + b"\0" * 100)
    with pytest.raises(ValueError):
        F.read_src(str(p))


@pytest.mark.gpu
def test_path_on_files_written_by_the_reference(cuda_ok, tmp_path):
    """Mesh and sources loaded from reference-written files, run through the
    device path (reference-order march, FP64 rates): the reference's own
    result on the same problem within 2e-6."""
    import torch
    from argot_b200 import _lib as L
    from argot_b200 import workload as W
    from argot_b200.pipeline import Problem
    wl = W.tiny(32, 12, seed=31)
    R = _loaded_ref(wl)
    mesh, prefix = str(tmp_path / "ref_000_000_000"), str(tmp_path / "ref")
    R.write_files(mesh, prefix)
    loaded = F.workload_from_files(mesh, prefix + "_src.dat", theta=wl.theta)
    pb = Problem(loaded)
    rates = pb.run(L.PRECISION_REFERENCE, L.RATE_EXACT_F64)
    torch.cuda.synchronize()
    got = rates.view(6, -1).cpu().numpy()
    R.zero_rates()
    R.run_range(0, 32 ** 3, True, want=())
    want = R.get_rates()
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() < 2e-6, rel.max(axis=1)
