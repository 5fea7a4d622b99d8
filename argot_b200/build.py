"""Builds libargot_b200.so in-tree for sm_100a with nvcc.

Every ``.cu`` file under ``argot_b200/csrc`` is compiled to an object in
``argot_b200/_build`` (in parallel, skipped when up to date) and linked into
``argot_b200/libargot_b200.so`` with the CUDA runtime linked statically, so
the library does not depend on which libcudart a host process already
loaded.

ARGOT's struct layouts and rate formula follow its preprocessor flags, so
the drop-in is also built for other flag sets: the sources that see the
reference's structs (those that include ``ref_layout.h``) are compiled again
with the set's flags and linked with the other objects into
``libargot_b200_<tag>.so``.  FLAGSETS lists the sets built by default (the
stock set of ARGOT's Makefile, -D__HYDROGEN_MOL__ -D__PHOTON_CONSERVING__,
among them); ``python -m argot_b200.build --flags "-D__HELIUM__ ..."`` builds
any other.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libargot_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _deps(src: str):
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    hdrs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return [src] + hdrs + [os.path.abspath(__file__)]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool, extra) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _stale(obj, _deps(src)):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise subprocess.CalledProcessError(r.returncode, cmd)
    if verbose and r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


# tag -> the reference's flags (the default library is helium + photon
# conserving)
FLAGSETS = {
    "h2_pc": ["-D__HYDROGEN_MOL__", "-D__PHOTON_CONSERVING__"],
    "he_h2_pc": ["-D__HELIUM__", "-D__HYDROGEN_MOL__", "-D__PHOTON_CONSERVING__"],
    "he": ["-D__HELIUM__"],
    "he_pc_cosmo": ["-D__HELIUM__", "-D__PHOTON_CONSERVING__", "-D__COSMOLOGICAL__"],
    "hi": [],
}


def flagset_tag(flags) -> str:
    """libargot_b200_<tag>.so for a list of -D flags"""
    f = set(flags)
    parts = [t for t, m in (("he", "-D__HELIUM__"), ("h2", "-D__HYDROGEN_MOL__"),
                            ("pc", "-D__PHOTON_CONSERVING__"), ("cosmo", "-D__COSMOLOGICAL__")) if m in f]
    if not ("-D__HELIUM__" in f or "-D__HYDROGEN_MOL__" in f):
        parts.insert(0, "hi")
    return "_".join(parts)


def flagset_lib(tag: str) -> str:
    return os.path.join(HERE, f"libargot_b200_{tag}.so")


def _layout_sources():
    return [s for s in sorted(glob.glob(os.path.join(CSRC, "*.cu")))
            if '#include "ref_layout.h"' in open(s).read()]


def build_flagset(flags, verbose: bool = False) -> str:
    """libargot_b200_<tag>.so: the library with its drop-in compiled for the
    reference flags `flags` (a list of -D options)."""
    tag = flagset_tag(flags)
    out = os.path.join(BUILD, "flags_" + tag)
    os.makedirs(out, exist_ok=True)
    layout = _layout_sources()
    extra = ["-DARGOT_FLAGSET_EXPLICIT", *flags]

    def comp(src):
        obj = os.path.join(out, os.path.basename(src) + ".o")
        if _stale(obj, _deps(src)):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, cmd)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, len(layout))) as ex:
        objs = list(ex.map(comp, layout))
    shared = [os.path.join(BUILD, os.path.basename(s) + ".o")
              for s in sorted(glob.glob(os.path.join(CSRC, "*.cu"))) if s not in layout]
    lib = flagset_lib(tag)
    if _stale(lib, objs + shared):
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, *shared, "-cudart", "static",
               "-Xlinker", "--no-undefined", "-Xlinker", "--exclude-libs,ALL",
               "-Xlinker", "-Bsymbolic", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose or ptxas_info, extra), srcs))
    if _stale(LIB, objs):
        # the static runtime's symbols stay private to this library
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static",
               "-Xlinker", "--no-undefined", "-Xlinker", "--exclude-libs,ALL",
               "-Xlinker", "-Bsymbolic", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_legacy(verbose)
    for flags in FLAGSETS.values():
        build_flagset(flags, verbose)
    return LIB


LEGACY_SRC = os.path.join(HERE, "legacy", "legacy.c")
LEGACY_LIB = os.path.join(HERE, "libargot_b200_legacy.so")


def build_legacy(verbose: bool = False) -> str:
    """libargot_b200_legacy.so: the older entry-point names
    (include/argot_b200_legacy.h) forwarded to libargot_b200.so, found next
    to it at run time."""
    deps = [LEGACY_SRC, LIB, os.path.join(INCLUDE, "argot_b200_legacy.h"), os.path.join(INCLUDE, "argot_b200.h")]
    if not _stale(LEGACY_LIB, deps):
        return LEGACY_LIB
    cmd = [os.environ.get("CC", "gcc"), "-O2", "-fPIC", "-shared", "-I" + INCLUDE, LEGACY_SRC, "-o", LEGACY_LIB,
           "-L" + HERE, "-l:libargot_b200.so", "-Wl,-rpath,$ORIGIN", "-Wl,--no-undefined"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LEGACY_LIB


if __name__ == "__main__":
    if "--flags" in sys.argv:
        print(build_flagset(sys.argv[sys.argv.index("--flags") + 1].split(), verbose="-v" in sys.argv))
    else:
        print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
