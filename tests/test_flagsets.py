"""The library built for ARGOT's other flag sets (the stock
-D__HYDROGEN_MOL__ build of src/Makefile, helium with H2, helium without
photon conservation, with the scale factor, hydrogen only): each build loads
without a GPU, exports the drop-in entry points, names its flag set, and its
struct layouts equal those of the reference compiled with the same flags."""
import ctypes as C

import numpy as np
import pytest

from flagset_util import layout, ref_flags, variant_lib

TAGS = ["h2_pc", "he_h2_pc", "he", "he_pc_cosmo", "hi"]
NAMES = {"h2_pc": "h2, photon conserving", "he_h2_pc": "helium+h2, photon conserving", "he": "helium",
         "he_pc_cosmo": "helium, photon conserving, cosmological", "hi": "hydrogen"}
DROPIN = ["calc_optical_depth_cuda", "calc_photoion_rate_cuda", "zero_out_photoion_rate_cuda",
          "accum_optical_depth", "smooth_photoion_rate", "argot_b200_abi_check", "argot_b200_last_error"]


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_library_loads_and_names_its_set(tag):
    lib = variant_lib(tag)
    assert lib.argot_b200_flagset().decode() == NAMES[tag]
    for name in DROPIN:
        assert hasattr(lib, name), name
    # the ART drop-in reads the helium layout: only the builds without H2
    # or the scale factor carry it
    assert hasattr(lib, "calc_diffuse_photon_radiation") == (tag == "he")


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_struct_sizes_match_reference(tag):
    lib = variant_lib(tag)
    mine = np.zeros(10, np.uint64)
    lib.argot_b200_struct_sizes(mine.ctypes.data)
    assert list(mine) == layout(tag).sizes()
    R = ref_flags(tag)
    theirs = np.zeros(10, np.uint64)
    R.refv_struct_sizes(theirs.ctypes.data)
    assert list(mine) == list(theirs)
    lib.argot_b200_abi_check.argtypes = [C.c_void_p, C.c_int]
    assert lib.argot_b200_abi_check(theirs.ctypes.data, 10) == 0


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_field_offsets_match_reference(tag):
    Lay = layout(tag)
    R = ref_flags(tag)
    o = np.zeros(12, np.uint64)
    R.refv_offsets(o.ctypes.data)
    mine = [Lay.PrimChem.fHI.offset, Lay.PrimChem.GammaHI.offset, Lay.FluidMesh.chem.offset,
            Lay.FluidMesh.prev_chem.offset, Lay.RaySegment.optical_depth_HI.offset,
            Lay.LightRay.ix_target.offset, Lay.LightRay.optical_depth_HI.offset,
            Lay.LightRayIO.optical_depth_HI.offset, Lay.RunParam.csect.offset, Lay.RunParam.nseg.offset,
            Lay.RunParam.nmesh_x_local.offset, Lay.RunParam.delta_x.offset]
    assert mine == list(o)


def test_flagset_tags_cover_the_build():
    from argot_b200 import abi, build
    assert sorted(abi.FLAGSETS) == sorted(TAGS)
    assert sorted(build.flagset_tag(f) for f in build.FLAGSETS.values()) == sorted(TAGS)
    from oracle import build as ob
    assert sorted(ob.REF_FLAGSETS) == sorted(TAGS)


@pytest.mark.parametrize("tag", TAGS)
def test_flagset_accum_optical_depth_host(tag):
    """accum_optical_depth (a host routine) carries every column of the set:
    ray r receives the columns of the segment with ray_indx r, rays without
    one get zero (one rank, accum_optical_depth.c:59-139)."""
    from argot_b200 import abi
    he, h2, _, _ = abi.FLAGSETS[tag]
    Lay = layout(tag)
    lib = variant_lib(tag)
    rng = np.random.default_rng(3)
    nray, nseg = 50, 40
    seg = np.zeros(nseg, dtype=np.dtype(Lay.RaySegment))
    seg["ray_indx"] = rng.permutation(nray)[:nseg]
    for c in Lay.columns:
        seg["optical_depth_" + c] = rng.uniform(0, 1, nseg).astype(np.float32)
    ray = np.zeros(nray, dtype=np.dtype(Lay.LightRay))
    for c in Lay.columns:
        ray["optical_depth_" + c] = -1.0
    run = Lay.RunParam()
    run.nray, run.nseg = nray, nseg
    lib.accum_optical_depth(ray.ctypes.data, seg.ctypes.data, C.addressof(run), None)
    assert lib.argot_b200_last_error() == 0
    for c in Lay.columns:
        want = np.zeros(nray, np.float32)
        want[seg["ray_indx"]] = seg["optical_depth_" + c]
        assert np.array_equal(ray["optical_depth_" + c], want), c
