"""ARGOT's on-disk formats for this path, so that a reference run's mesh
and sources can be loaded as inputs and results written back.

* Source list ``<prefix>_src.dat`` (output_data.c:59-73, input_data.c:
  165-223): uint64 nsrc, struct freq_param, nsrc x struct radiation_src
  (type, param, x, y, z, 256 FP64 photon rates per bin).
* Mesh dump ``<prefix>_<rx>_<ry>_<rz>`` of one rank (output_data.c:14-57,
  input_data.c:48-163): struct run_param, then per cell (z fastest) a
  struct fluid_mesh_io (dens, eneg, momx, momy, momz, uene, pot, chem).

The structs are the byte-identical mirrors of ``abi.py`` (the reference's
default flag set: helium, no H2).  A reader of the reference checks the
header's mesh sizes, rank counts, species and channel numbers against its
build; ``write_mesh`` fills them for a single-rank mesh.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .workload import Workload

NSPECIES = 5   # HI, HII, HeI, HeII, HeIII (run_param.h:84-98 with __HELIUM__)
NCHANNEL = 3   # HI, HeI, HeII

SRC_DTYPE = np.dtype(abi.RadiationSrc)
MESH_DTYPE = np.dtype(abi.FluidMeshIO)


def read_src(path: str):
    """(freq_param bytes, structured array of radiation_src)."""
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(8), np.uint64)[0])
        freq = f.read(C.sizeof(abi.FreqParam))
        src = np.frombuffer(f.read(n * SRC_DTYPE.itemsize), SRC_DTYPE)
    if len(src) != n or len(freq) != C.sizeof(abi.FreqParam):
        raise ValueError(f"{path}: truncated source file")
    return freq, src.copy()


def write_src(path: str, src_type, src_param, src_pos, photon_rate, freq: bytes | None = None):
    """A source file readable by the reference (freq: the freq_param bytes
    to store; default the reference's frequency grid of this library)."""
    n = len(src_type)
    rec = np.zeros(n, SRC_DTYPE)
    rec["type"] = np.asarray(src_type, np.int32)
    rec["param"] = np.asarray(src_param, np.float32)
    pos = np.asarray(src_pos, np.float32).reshape(n, 3)
    rec["xpos"], rec["ypos"], rec["zpos"] = pos[:, 0], pos[:, 1], pos[:, 2]
    rec["photon_rate"] = np.asarray(photon_rate, np.float64).reshape(n, -1)
    if freq is None:
        freq = bytes(default_freq_param())
    with open(path, "wb") as f:
        f.write(np.uint64(n).tobytes())
        f.write(freq)
        f.write(rec.tobytes())


def default_freq_param() -> abi.FreqParam:
    """struct freq_param as setup_freq_param (source.c:38-53) fills it."""
    from .pipeline import tables
    nu, _ = tables()
    fp = abi.FreqParam()
    fp.log_nu_min, fp.log_nu_max = 0.0, 1.5
    fp.dlog_nu = 1.5 / 256
    for i in range(256):
        fp.nu[i] = nu[i]
    return fp


def read_mesh(path: str):
    """(run_param, structured array of fluid_mesh_io) of one rank's dump."""
    hdr = abi.RunParam()
    with open(path, "rb") as f:
        raw = f.read(C.sizeof(abi.RunParam))
        if len(raw) != C.sizeof(abi.RunParam):
            raise ValueError(f"{path}: truncated header")
        C.memmove(C.addressof(hdr), raw, len(raw))
        n = hdr.nmesh_x_local * hdr.nmesh_y_local * hdr.nmesh_z_local
        cells = np.frombuffer(f.read(n * MESH_DTYPE.itemsize), MESH_DTYPE)
    if len(cells) != n:
        raise ValueError(f"{path}: truncated mesh ({len(cells)} of {n} cells)")
    return hdr, cells.copy()


def mesh_header(edge: int, lunit: float, denstonh: float) -> abi.RunParam:
    """run_param of a single-rank edge^3 unit-box mesh with the fields a
    reader checks (input_data.c:48-110)."""
    h = abi.RunParam()
    h.helium_flag, h.ngrid_nu, h.mpi_rank, h.mpi_nproc = 1, 256, 0, 1
    h.nnode_x = h.nnode_y = h.nnode_z = 1
    h.lunit, h.denstonh = lunit, denstonh
    h.anow = 1.0
    h.nspecies, h.nchannel = NSPECIES, NCHANNEL
    h.xmax = h.ymax = h.zmax = 1.0
    h.xmax_local = h.ymax_local = h.zmax_local = 1.0
    h.nmesh_x_total = h.nmesh_y_total = h.nmesh_z_total = edge
    h.nmesh_x_local = h.nmesh_y_local = h.nmesh_z_local = edge
    d = float(np.float32(1.0) / np.float32(edge))
    h.delta_x = h.delta_y = h.delta_z = d
    h.freq = default_freq_param()
    return h


def write_mesh(path: str, hdr: abi.RunParam, dens, fHI, fHeI, fHeII, rates6=None):
    """A one-rank mesh dump: the ionisation state from fHI, fHeI, fHeII
    (fHII = 1 - fHI, fHeIII = 1 - fHeI - fHeII) and, when given, the six
    rate fields in chem (Gamma and Heat of HI, HeI, HeII); other fields 0."""
    n = len(dens)
    rec = np.zeros(n, MESH_DTYPE)
    rec["dens"] = dens
    chem = rec["chem"]
    chem["fHI"], chem["fHII"] = fHI, np.float32(1.0) - np.asarray(fHI, np.float32)
    chem["fHeI"], chem["fHeII"] = fHeI, fHeII
    chem["fHeIII"] = np.float32(1.0) - np.asarray(fHeI, np.float32) - np.asarray(fHeII, np.float32)
    if rates6 is not None:
        r = np.asarray(rates6, np.float32).reshape(6, n)
        for j, k in enumerate(("GammaHI", "GammaHeI", "GammaHeII", "HeatHI", "HeatHeI", "HeatHeII")):
            chem[k] = r[j]
    rec["chem"] = chem
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(rec.tobytes())


def workload_from_files(mesh_path: str, src_path: str, theta: float = 0.5, name: str | None = None) -> Workload:
    """A single-rank unit-box mesh and its sources as a Workload (the
    photon rates per bin taken from the file)."""
    hdr, cells = read_mesh(mesh_path)
    e = hdr.nmesh_x_local
    if (hdr.nmesh_y_local, hdr.nmesh_z_local) != (e, e) or hdr.mpi_nproc != 1:
        raise ValueError("only single-rank cubic meshes are supported")
    _, src = read_src(src_path)
    chem = cells["chem"]
    pos = np.stack([src["xpos"], src["ypos"], src["zpos"]], 1).astype(np.float32)
    spec = np.ascontiguousarray(src["photon_rate"], np.float64)
    return Workload(name=name or f"file{e}_src{len(src)}", edge=e,
                    dens=np.ascontiguousarray(cells["dens"], np.float32),
                    fHI=np.ascontiguousarray(chem["fHI"], np.float32),
                    fHeI=np.ascontiguousarray(chem["fHeI"], np.float32),
                    fHeII=np.ascontiguousarray(chem["fHeII"], np.float32),
                    src_pos=pos, src_rate=spec.sum(1), src_type=np.asarray(src["type"], np.int32),
                    src_param=np.asarray(src["param"], np.float32), theta=theta, lunit=hdr.lunit,
                    denstonh=hdr.denstonh, notes=f"read from {mesh_path} and {src_path}",
                    src_spectra=spec)
