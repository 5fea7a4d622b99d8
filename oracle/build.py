"""Build recipes for the checkers and baselines (test infrastructure only).

1. O1, the parity oracle: ARGOT's own hot-path C, compiled unmodified from the
   reference tree, one shared library per mesh edge, into
   ``oracle/_ref/libargot_ref_n<EDGE>.so``.
2. The reference's GPU entry points of this path compiled for sm_100a
   (``build_ref_gpu``, ``oracle/_ref/libargot_refgpu_n<EDGE>.so``): the
   reference-GPU baseline of the benchmark.
3. The restatement (``oracle/argot_oracle.c``, ref-order FP32/FP64 functions and
   the FP64 precision oracle) into ``oracle/_build/libargot_oracle.so``.
4. O1 for ARGOT's other flag sets (``build_ref_flags``: the hot-path sources
   with the stock ``-D__HYDROGEN_MOL__`` set, helium + H2, no photon
   conservation, the scale factor, hydrogen only; driver
   ``oracle/ref_flags_driver.c``) into
   ``oracle/_ref/libargot_ref_flags_<tag>_n16.so``.

Both directories are git-ignored; the built libraries travel with the working
tree.  Nothing in the product path (the ``argot_b200`` package) loads them.

The reference fixes the local mesh size at compile time (``NMESH_*_TOTAL`` and
``NNODE_*`` in ``src/run_param.h:22-69``).  For each edge N the recipe writes a
copy of ``run_param.h`` with only those two settings changed (N^3 cells, one
rank) to ``oracle/_ref/inc_N/`` and compiles the reference sources where they
lie, with ``-I<inc_N> -I-`` so that the patched header is found before the
original one (``-I-`` also disables the lookup of quoted includes in the
including file's own directory).  Sources compiled: exactly the hot path and
what it calls:

  calc_optical_depth.c      (A1, CPU march)
  accum_optical_depth.c     (A2, stitching)
  calc_photoion_rate.c      (A3/A4, rate integral, zeroing)
  calc_ray_segment.c, assign_ray_segment.c, setup_light_ray_tree.c
                            (ray construction feeding the path)
  source.c, cross_section.c, prim_chem/cross_section.c
                            (A5 tables)
  mpi_rank.c, timing.c      (helpers)
  smooth_photoion_rate.c, output_data.c, input_data.c, make_directory.c
                            (smoothing, file formats)
  diffuse_photon/*.c        (ART diffuse radiation, CPU build)

plus files of ours: ``oracle/shim/mpi.h`` (single-rank MPI),
``oracle/shim/chealpix.h`` (HEALPix pix2ang_ring, which chealpix would
provide) and ``oracle/ref_driver.c`` (flat-array glue).  ``-fgnu89-inline``
gives the diffuse sources' plain ``inline`` functions an external
definition, as the compilers the reference was written for did.  Flags follow the reference's
``src/Makefile`` switches for this path (``-D__HELIUM__ -D__PHOTON_CONSERVING__
-D__RADIATION_TRANSFER__ -D__ARGOT_PROFILE__``, and the Makefile's default
``-D__HEATCOOL__``, which on these sources only sets the diffuse-radiation
step-function range), ``-O2`` without
``-ffast-math`` (the parity build); ``--fast-math`` adds the reference's own
``-ffast-math`` for the spread study.  ``-ffp-contract=off`` pins IEEE
single-operation rounding (the x86-64 baseline target has no FMA anyway).
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
ORC_OUT = os.path.join(HERE, "_build")
# ARGOT's source tree: $ARGOT_REFERENCE, else a checkout named ``reference``
# beside this repository
DEFAULT_REF = os.environ.get("ARGOT_REFERENCE",
                             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

SOURCES = [
    "calc_optical_depth.c",
    "accum_optical_depth.c",
    "calc_photoion_rate.c",
    "calc_ray_segment.c",
    "assign_ray_segment.c",
    "setup_light_ray_tree.c",
    "source.c",
    "cross_section.c",
    "prim_chem/cross_section.c",
    "mpi_rank.c",
    "timing.c",
    "smooth_photoion_rate.c",
    "output_data.c",
    "input_data.c",
    "make_directory.c",
    # ART diffuse radiation (CPU build)
    "diffuse_photon/set_angle.c",
    "diffuse_photon/set_start_pos.c",
    "diffuse_photon/set_step_func_factor.c",
    "diffuse_photon/setup_diffuse.c",
    "diffuse_photon/init_hd_param.c",
    "diffuse_photon/ray_tracing.c",
    "diffuse_photon/calc_rmesh_data.c",
    "diffuse_photon/calc_GH_tot.c",
    "diffuse_photon/calc_diffuse_photon_radiation.c",
    "diffuse_photon/operation_mpi_window.c",
    "diffuse_photon/diffuse_photon_mpi.c",
]

# 19: a ragged mesh (no axis a multiple of the 2x4x4 target blocks); 24: an
# even edge that is no power of two (the reference's ART pass groups its
# start rays 2x2, set_start_pos.c:88, so it needs even edges)
EDGES = (16, 19, 24, 32, 48, 64, 96, 128, 192, 256)
# the reference's GPU build: the test problem and the benchmark workloads
GPU_EDGES = (16, 64, 128, 192, 256)

FLAGS = ["-D__HELIUM__", "-D__PHOTON_CONSERVING__", "-D__RADIATION_TRANSFER__",
         "-D__ARGOT_PROFILE__", "-D__HEATCOOL__"]


def _cc() -> str:
    return os.environ.get("ARGOT_CC", "gcc")


def patched_run_param(src_text: str, edge: int) -> str:
    """run_param.h with an N^3 single-rank mesh; nothing else changes."""
    t = re.sub(r"#define\s+NMESH_([XYZ])_TOTAL\s+\(\d+\)",
               lambda m: f"#define NMESH_{m.group(1)}_TOTAL ({edge})", src_text)
    t = re.sub(r"#define\s+NNODE_([XYZ])\s+\(\d+\)",
               lambda m: f"#define NNODE_{m.group(1)} (1)", t)
    return t


def ref_lib_path(edge: int, fast_math: bool = False, isolated: bool = False) -> str:
    tag = ("_fm" if fast_math else "") + ("_iso" if isolated else "")
    return os.path.join(REF_OUT, f"libargot_ref_n{edge}{tag}.so")


def oracle_lib_path() -> str:
    return os.path.join(ORC_OUT, "libargot_oracle.so")


def reference_available(ref: str = DEFAULT_REF) -> bool:
    return os.path.isdir(os.path.join(ref, "src"))


def build_ref(edge: int, ref: str = DEFAULT_REF, fast_math: bool = False,
              verbose: bool = False, isolated: bool = False) -> str:
    """isolated: the reference Makefile's default `isolated = yes`
    (-D__ISOLATED__), which only changes mpi_rank.c on this path: a missing
    neighbour rank instead of the periodic image."""
    src_dir = os.path.join(ref, "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference sources not found at {src_dir}")
    inc = os.path.join(REF_OUT, f"inc_{edge}")
    os.makedirs(inc, exist_ok=True)
    with open(os.path.join(src_dir, "run_param.h")) as f:
        text = patched_run_param(f.read(), edge)
    with open(os.path.join(inc, "run_param.h"), "w") as f:
        f.write(text)
    out = ref_lib_path(edge, fast_math, isolated)
    cmd = [_cc(), "-O2", "-std=gnu99", "-fgnu89-inline", "-fopenmp", "-fPIC", "-shared", "-w",
           "-fno-strict-aliasing", "-ffp-contract=off"]
    if fast_math:
        cmd.append("-ffast-math")
    cmd += FLAGS
    if isolated:
        cmd.append("-D__ISOLATED__")
    cmd += ["-I" + inc, "-I-", "-I" + os.path.join(HERE, "shim"),
            "-I" + src_dir, "-I" + os.path.join(src_dir, "prim_chem"),
            "-I" + os.path.join(src_dir, "diffuse_photon")]
    cmd += [os.path.join(src_dir, s) for s in SOURCES]
    cmd += [os.path.join(HERE, "ref_driver.c"), "-o", out, "-lm",
            "-Wl,--no-undefined"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise subprocess.CalledProcessError(r.returncode, cmd)
    return out


# the hot-path sources a flag-set build needs (the rays are made by the test)
FLAG_SOURCES = ["calc_optical_depth.c", "calc_photoion_rate.c", "source.c", "cross_section.c",
                "prim_chem/cross_section.c", "mpi_rank.c", "timing.c", "smooth_photoion_rate.c"]
# tag -> the reference flags of the flag sets the library is also built for
# (argot_b200/build.py FLAGSETS); every build is -D__ISOLATED__, as the
# reference Makefile's default
REF_FLAGSETS = {
    "h2_pc": ["-D__HYDROGEN_MOL__", "-D__PHOTON_CONSERVING__"],
    "he_h2_pc": ["-D__HELIUM__", "-D__HYDROGEN_MOL__", "-D__PHOTON_CONSERVING__"],
    "he": ["-D__HELIUM__"],
    "he_pc_cosmo": ["-D__HELIUM__", "-D__PHOTON_CONSERVING__", "-D__COSMOLOGICAL__"],
    "hi": [],
}


def ref_flags_lib_path(tag: str, edge: int) -> str:
    return os.path.join(REF_OUT, f"libargot_ref_flags_{tag}_n{edge}.so")


def build_ref_flags(tag: str, edge: int = 16, ref: str = DEFAULT_REF, verbose: bool = False) -> str:
    """ARGOT's own calc_optical_depth.c / calc_photoion_rate.c /
    smooth_photoion_rate.c and their tables, compiled unmodified with the
    flag set REF_FLAGSETS[tag] (plus -D__RADIATION_TRANSFER__
    -D__ARGOT_PROFILE__ -D__ISOLATED__) and ref_flags_driver.c into
    oracle/_ref/libargot_ref_flags_<tag>_n<EDGE>.so."""
    src_dir = os.path.join(ref, "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference sources not found at {src_dir}")
    inc = os.path.join(REF_OUT, f"inc_{edge}")
    os.makedirs(inc, exist_ok=True)
    with open(os.path.join(src_dir, "run_param.h")) as f:
        text = patched_run_param(f.read(), edge)
    with open(os.path.join(inc, "run_param.h"), "w") as f:
        f.write(text)
    out = ref_flags_lib_path(tag, edge)
    cmd = [_cc(), "-O2", "-std=gnu99", "-fgnu89-inline", "-fopenmp", "-fPIC", "-shared", "-w",
           "-fno-strict-aliasing", "-ffp-contract=off", *REF_FLAGSETS[tag],
           "-D__RADIATION_TRANSFER__", "-D__ARGOT_PROFILE__", "-D__HEATCOOL__", "-D__ISOLATED__",
           "-I" + inc, "-I-", "-I" + os.path.join(HERE, "shim"),
           "-I" + src_dir, "-I" + os.path.join(src_dir, "prim_chem")]
    cmd += [os.path.join(src_dir, s) for s in FLAG_SOURCES]
    cmd += [os.path.join(HERE, "ref_flags_driver.c"), "-o", out, "-lm", "-Wl,--no-undefined"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise subprocess.CalledProcessError(r.returncode, cmd)
    return out


def refgpu_lib_path(edge: int) -> str:
    return os.path.join(REF_OUT, f"libargot_refgpu_n{edge}.so")


# the reference's GPU entry points for this path and their pinned allocators
GPU_SOURCES = ["calc_optical_depth_cuda.cu", "calc_photoion_rate_cuda.cu", "allocate_pinned_segment.cu"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def build_ref_gpu(edge: int, ref: str = DEFAULT_REF, verbose: bool = False) -> str:
    """ARGOT's own GPU entry points for this path (GPU_SOURCES), compiled
    unmodified for sm_100a with the reference Makefile's nvcc flags
    (``src/Makefile:208``: ``-use_fast_math -O3``), linked with the CPU
    reference (SOURCES, which build the rays) and our glue
    (``ref_driver.c``, ``ref_gpu_driver.cu``) into
    ``oracle/_ref/libargot_refgpu_n<EDGE>.so``.

    nvcc cannot take ``-I-`` (CUDA's own headers need their directory's
    quoted includes), so the reference's ``src/`` is copied to a temporary
    directory outside the repository, its ``run_param.h`` replaced by the
    patched one, compiled there and deleted: nothing of the reference is
    kept but the library."""
    src_dir = os.path.join(ref, "src")
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference sources not found at {src_dir}")
    os.makedirs(REF_OUT, exist_ok=True)
    out = refgpu_lib_path(edge)
    tmp = tempfile.mkdtemp(prefix="argot_refgpu_")
    try:
        tsrc = os.path.join(tmp, "src")
        shutil.copytree(src_dir, tsrc, ignore=shutil.ignore_patterns("*.o", "*.a", "*.so"))
        with open(os.path.join(src_dir, "run_param.h")) as f:
            text = patched_run_param(f.read(), edge)
        with open(os.path.join(tsrc, "run_param.h"), "w") as f:
            f.write(text)
        inc = ["-I" + os.path.join(HERE, "shim"), "-I" + tsrc, "-I" + os.path.join(tsrc, "prim_chem"),
               "-I" + os.path.join(tsrc, "diffuse_photon")]
        objs = []

        def run(cmd):
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stderr)
                raise subprocess.CalledProcessError(r.returncode, cmd)

        for i, name in enumerate(SOURCES + ["ref_driver.c"]):
            path = os.path.join(HERE, name) if name == "ref_driver.c" else os.path.join(tsrc, name)
            o = os.path.join(tmp, f"c{i}.o")
            run([_cc(), "-O2", "-std=gnu99", "-fgnu89-inline", "-fopenmp", "-fPIC", "-w", "-fno-strict-aliasing",
                 "-ffp-contract=off", *FLAGS, *inc, "-c", path, "-o", o])
            objs.append(o)
        gpu_flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-use_fast_math", "-O3",
                     "-Xcompiler", "-fPIC", "-w", *FLAGS, "-D__USE_GPU__", "-D__USE_GPU_ARGOT__", *inc]
        for i, name in enumerate(GPU_SOURCES + ["ref_gpu_driver.cu"]):
            path = os.path.join(HERE, name) if name == "ref_gpu_driver.cu" else os.path.join(tsrc, name)
            o = os.path.join(tmp, f"g{i}.o")
            run([_nvcc(), *gpu_flags, "-c", path, "-o", o])
            objs.append(o)
        run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out, *objs,
             "-cudart", "static", "-Xcompiler", "-fopenmp", "-Xlinker", "--no-undefined",
             "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-Bsymbolic", "-lm",
             "-lpthread", "-ldl", "-lrt"])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def build_oracle(verbose: bool = False) -> str:
    os.makedirs(ORC_OUT, exist_ok=True)
    out = oracle_lib_path()
    cmd = [_cc(), "-O2", "-std=gnu99", "-fopenmp", "-fPIC", "-shared", "-Wall",
           "-ffp-contract=off", os.path.join(HERE, "argot_oracle.c"), "-o", out,
           "-lm", "-Wl,--no-undefined"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


def build_all(edges=EDGES, ref: str = DEFAULT_REF, verbose: bool = False):
    """Restatement always; the reference builds when its sources are here."""
    built = [build_oracle(verbose)]
    if reference_available(ref):
        for e in edges:
            built.append(build_ref(e, ref, False, verbose))
        built.append(build_ref(64, ref, True, verbose))
        built.append(build_ref(16, ref, False, verbose, isolated=True))
        built.append(build_ref(32, ref, False, verbose, isolated=True))
        for tag in REF_FLAGSETS:
            built.append(build_ref_flags(tag, 16, ref, verbose))
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(max_workers=min(len(GPU_EDGES), os.cpu_count() or 1)) as ex:
            built += list(ex.map(lambda e: build_ref_gpu(e, ref, verbose), GPU_EDGES))
    return built


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__,
                                formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--ref", default=DEFAULT_REF)
    p.add_argument("--edges", default=",".join(map(str, EDGES)))
    p.add_argument("-v", "--verbose", action="store_true")
    a = p.parse_args(argv)
    for path in build_all([int(x) for x in a.edges.split(",") if x], a.ref, a.verbose):
        print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
