"""ctypes mirrors of the ARGOT structs that cross the drop-in boundary
(reference flag set: helium, photon conserving, no H2; NGRID_NU=256,
NSEG_PER_RAY=5, NMAX_CUDA_DEV=4).  Field order follows src/radiation.h,
src/fluid.h, src/source.h, src/prim_chem/chemistry.h, src/run_param.h and
src/cuda_mem_space.h; the sizes are asserted by the test suite against both
the reference compiled here and libargot_b200's own view.

Used by callers that drive the drop-in entry points from Python (the tests
and the reference-facing end-to-end path of bench.py).
"""
from __future__ import annotations

import ctypes as C

NGRID_NU = 256
NSEG_PER_RAY = 5
NMAX_CUDA_DEV = 4


class PrimChem(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("wmol", "felec", "fHI", "fHII", "fHeI", "fHeII", "fHeIII", "GammaHI", "HeatHI",
                 "GammaHeI", "GammaHeII", "HeatHeI", "HeatHeII")]


class FluidMesh(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("dens", "eneg", "momx", "momy", "momz", "uene", "duene", "durad", "etrp", "pot",
                 "dens_prev")] + [("chem", PrimChem), ("prev_chem", PrimChem),
                                  ("prev_uene", C.c_float), ("under_shock", C.c_short),
                                  ("high_mach", C.c_short)]


class FluidMeshIO(C.Structure):
    """struct fluid_mesh_io (fluid.h:118-125): one cell of a mesh dump"""
    _fields_ = [(n, C.c_float) for n in ("dens", "eneg", "momx", "momy", "momz", "uene", "pot")] + \
               [("chem", PrimChem)]


class RadiationSrc(C.Structure):
    _fields_ = [("type", C.c_int), ("param", C.c_float), ("xpos", C.c_float),
                ("ypos", C.c_float), ("zpos", C.c_float),
                ("photon_rate", C.c_double * NGRID_NU)]


class RaySegment(C.Structure):
    _fields_ = [("ray_indx", C.c_uint64), ("local_rank", C.c_int), ("target_rank", C.c_int),
                ("xpos_start", C.c_float), ("ypos_start", C.c_float), ("zpos_start", C.c_float),
                ("xpos_end", C.c_float), ("ypos_end", C.c_float), ("zpos_end", C.c_float),
                ("optical_depth_HI", C.c_float), ("optical_depth_HeI", C.c_float),
                ("optical_depth_HeII", C.c_float)]


class LightRay(C.Structure):
    _fields_ = [("src", RadiationSrc), ("num_segment", C.c_int),
                ("segment", RaySegment * NSEG_PER_RAY),
                ("ix_target", C.c_int), ("iy_target", C.c_int), ("iz_target", C.c_int),
                ("optical_depth_HI", C.c_float), ("optical_depth_HeI", C.c_float),
                ("optical_depth_HeII", C.c_float)]


class LightRayIO(C.Structure):
    _fields_ = [("src", RadiationSrc),
                ("ix_target", C.c_int), ("iy_target", C.c_int), ("iz_target", C.c_int),
                ("optical_depth_HI", C.c_float), ("optical_depth_HeI", C.c_float),
                ("optical_depth_HeII", C.c_float)]


class CrossSection(C.Structure):
    _fields_ = [("csect_HI", C.c_float), ("csect_HeI", C.c_float), ("csect_HeII", C.c_float)]


class FreqParam(C.Structure):
    _fields_ = [("log_nu_min", C.c_double), ("log_nu_max", C.c_double),
                ("dlog_nu", C.c_double), ("nu", C.c_double * NGRID_NU)]


class PhotoionRate(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("GammaHI", "HeatHI", "GammaHeI", "GammaHeII", "HeatHeI", "HeatHeII")]


class Cosmology(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("omega_m", "omega_v", "omega_b", "omega_nu", "hubble", "tend")]


class RunParam(C.Structure):
    _fields_ = ([("model_name", C.c_void_p), ("proc_file", C.c_void_p), ("diag_file", C.c_void_p),
                 ("err_file", C.c_void_p)]
                + [(n, C.c_int) for n in ("helium_flag", "hydrogen_mol_flag", "cosmology_flag",
                                          "ngrid_nu", "mpi_rank", "mpi_nproc", "rank_x", "rank_y",
                                          "rank_z", "nnode_x", "nnode_y", "nnode_z")]
                + [(n, C.c_double) for n in ("lunit", "munit", "tunit", "eunit", "denstonh",
                                             "uenetok", "masstonh")]
                + [(n, C.c_float) for n in ("anow", "tnow", "znow", "hnow")]
                + [("cosm", Cosmology), ("tend", C.c_float), ("dtime", C.c_float),
                   ("freq", FreqParam), ("csect", CrossSection * NGRID_NU)]
                + [(n, C.c_int) for n in ("nspecies", "nchannel", "step", "output_indx", "noutput")]
                + [("output_timing", C.c_void_p)]
                + [(n, C.c_uint64) for n in ("nsrc", "nray", "nseg")]
                + [(n, C.c_float) for n in ("xmin", "ymin", "zmin", "xmax", "ymax", "zmax",
                                            "xmin_local", "ymin_local", "zmin_local",
                                            "xmax_local", "ymax_local", "zmax_local")]
                + [(n, C.c_int) for n in ("nmesh_x_total", "nmesh_y_total", "nmesh_z_total",
                                          "nmesh_x_local", "nmesh_y_local", "nmesh_z_local")]
                + [(n, C.c_float) for n in ("delta_x", "delta_y", "delta_z", "theta_crit")]
                + [("nmesh_per_loop", C.c_int)])


class CudaParam(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("num_cuda_dev", "nmesh_per_dev", "cuda_nblock",
                                        "max_thread_dimx", "max_block_dimx")]
                + [("strm", C.c_int64 * NMAX_CUDA_DEV), ("diffuse_strm", C.c_int64 * NMAX_CUDA_DEV)])


class CudaMemSpace(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("mesh_dev", "this_run_dev", "freq_dev", "segment_dev",
                                          "rate_dev", "chem_updated", "ray_IO_dev",
                                          "optical_depth_dev", "dtime_dev", "diff_chem_dev",
                                          "diff_uene_dev")]


STRUCTS = [RaySegment, LightRay, LightRayIO, RadiationSrc, FluidMesh, PrimChem, RunParam,
           CrossSection, FreqParam, PhotoionRate]


def sizes():
    return [C.sizeof(s) for s in STRUCTS]


def offsets():
    """Same order as ref_struct_offsets in oracle/ref_driver.c."""
    o = C.Structure
    return [RaySegment.ray_indx.offset, RaySegment.xpos_start.offset,
            RaySegment.optical_depth_HI.offset, LightRay.num_segment.offset,
            LightRay.segment.offset, LightRay.ix_target.offset, LightRay.optical_depth_HI.offset,
            LightRayIO.ix_target.offset, LightRayIO.optical_depth_HI.offset,
            RadiationSrc.photon_rate.offset, FluidMesh.chem.offset, FluidMesh.prev_chem.offset,
            PrimChem.fHI.offset, PrimChem.fHeI.offset, PrimChem.GammaHI.offset,
            PrimChem.HeatHeII.offset, RunParam.lunit.offset, RunParam.denstonh.offset,
            RunParam.freq.offset, RunParam.csect.offset, RunParam.nsrc.offset,
            RunParam.nray.offset, RunParam.nseg.offset, RunParam.xmin.offset,
            RunParam.xmin_local.offset, RunParam.nmesh_x_total.offset,
            RunParam.nmesh_x_local.offset, RunParam.delta_x.offset, RunParam.theta_crit.offset,
            RunParam.nmesh_per_loop.offset, RunParam.rank_x.offset, RunParam.anow.offset]


# ---------------------------------------------------------------- flag sets
def column_names(helium: bool, hydrogen_mol: bool):
    """The optical_depth_* columns of a segment / ray in the reference's
    order (src/radiation.h:23-83)."""
    return (["HI"] + (["HeI", "HeII"] if helium else [])
            + (["HM", "H2I", "H2II"] if hydrogen_mol else []))


def rate_names(helium: bool, hydrogen_mol: bool):
    """The Gamma / Heat fields of struct prim_chem from GammaHI on
    (src/prim_chem/chemistry.h:41-63)."""
    return (["GammaHI", "HeatHI"]
            + (["GammaHeI", "GammaHeII", "HeatHeI", "HeatHeII"] if helium else [])
            + (["GammaHM", "GammaH2I_I", "GammaH2I_II", "GammaH2II_I", "GammaH2II_II",
                "HeatHM", "HeatH2I_I", "HeatH2I_II", "HeatH2II_I", "HeatH2II_II"] if hydrogen_mol else []))


def channel_names(helium: bool, hydrogen_mol: bool):
    """The csect_* fields of struct cross_section (src/cross_section.h:7-20)."""
    return (["HI"] + (["HeI", "HeII"] if helium else [])
            + (["HM", "H2I_I", "H2II_I", "H2II_II"] if hydrogen_mol else []))


def make_layout(helium: bool = True, hydrogen_mol: bool = False):
    """ctypes mirrors of the structs for another flag set of the reference:
    the fields that -D__HELIUM__ and -D__HYDROGEN_MOL__ add sit where the
    reference headers put them.  Returns a namespace with PrimChem,
    FluidMesh, RaySegment, LightRay, LightRayIO, CrossSection, PhotoionRate,
    RunParam, STRUCTS (the order of argot_b200_struct_sizes) and the column /
    rate / channel names."""
    import types
    cols = column_names(helium, hydrogen_mol)
    rates = rate_names(helium, hydrogen_mol)
    chans = channel_names(helium, hydrogen_mol)
    f = C.c_float

    class PrimChemV(C.Structure):
        _fields_ = ([(n, f) for n in ("wmol", "felec", "fHI", "fHII")]
                    + ([(n, f) for n in ("fH2I", "fH2II", "fHM")] if hydrogen_mol else [])
                    + ([(n, f) for n in ("fHeI", "fHeII", "fHeIII")] if helium else [])
                    + [(n, f) for n in rates])

    class FluidMeshV(C.Structure):
        _fields_ = [(n, f) for n in
                    ("dens", "eneg", "momx", "momy", "momz", "uene", "duene", "durad", "etrp", "pot",
                     "dens_prev")] + [("chem", PrimChemV), ("prev_chem", PrimChemV),
                                      ("prev_uene", f), ("under_shock", C.c_short),
                                      ("high_mach", C.c_short)]

    class RaySegmentV(C.Structure):
        _fields_ = ([("ray_indx", C.c_uint64), ("local_rank", C.c_int), ("target_rank", C.c_int)]
                    + [(n, f) for n in ("xpos_start", "ypos_start", "zpos_start",
                                        "xpos_end", "ypos_end", "zpos_end")]
                    + [("optical_depth_" + c, f) for c in cols])

    class LightRayV(C.Structure):
        _fields_ = ([("src", RadiationSrc), ("num_segment", C.c_int),
                     ("segment", RaySegmentV * NSEG_PER_RAY),
                     ("ix_target", C.c_int), ("iy_target", C.c_int), ("iz_target", C.c_int)]
                    + [("optical_depth_" + c, f) for c in cols])

    class LightRayIOV(C.Structure):
        _fields_ = ([("src", RadiationSrc),
                     ("ix_target", C.c_int), ("iy_target", C.c_int), ("iz_target", C.c_int)]
                    + [("optical_depth_" + c, f) for c in cols])

    class CrossSectionV(C.Structure):
        _fields_ = [("csect_" + c, f) for c in chans]

    class PhotoionRateV(C.Structure):
        _fields_ = [(n, f) for n in rates]

    run_fields = []
    for name, typ in RunParam._fields_:
        run_fields.append((name, CrossSectionV * NGRID_NU if name == "csect" else typ))

    class RunParamV(C.Structure):
        _fields_ = run_fields

    ns = types.SimpleNamespace(
        PrimChem=PrimChemV, FluidMesh=FluidMeshV, RaySegment=RaySegmentV, LightRay=LightRayV,
        LightRayIO=LightRayIOV, CrossSection=CrossSectionV, PhotoionRate=PhotoionRateV,
        RunParam=RunParamV, RadiationSrc=RadiationSrc, FreqParam=FreqParam,
        columns=cols, rates=rates, channels=chans)
    ns.STRUCTS = [RaySegmentV, LightRayV, LightRayIOV, RadiationSrc, FluidMeshV, PrimChemV, RunParamV,
                  CrossSectionV, FreqParam, PhotoionRateV]
    ns.sizes = lambda: [C.sizeof(s) for s in ns.STRUCTS]
    return ns


# the flag sets the library is also built for: tag -> (helium, H2, photon
# conserving, cosmological); the default library is helium + photon conserving
FLAGSETS = {
    "h2_pc": (False, True, True, False),
    "he_h2_pc": (True, True, True, False),
    "he": (True, False, False, False),
    "he_pc_cosmo": (True, False, True, True),
    "hi": (False, False, False, False),
}
