"""Builds libcetagpu.so (sm_100a) in-tree with nvcc.

The library is a plain C-ABI shared object (include/cetasim_gpu.h); nothing in
it depends on PyTorch.  Usage: ``python -m cetasim_b200.build`` or
``cetasim_b200.build.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcetagpu.so")

SOURCES = ["capi.cu", "kernels.cu", "kernels_sr.cu", "kernels_ion.cu", "surrogate.cu", "shard.cu",
           "cbm.cu", "beam_loading.cu", "bbi.cu", "sc.cu", "faddeeva_table.cpp", "input_settings.cpp", "rw_wake.cpp"]
HEADERS = ["cg_common.cuh", "faddeeva.cuh", "be_field.cuh", "track_math.cuh", "cg_internal.h",
           "kernels.cuh", "umma.cuh", "surrogate.cuh", "rw_wake.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--compiler-options", "-fPIC",
    "-Xptxas", "-O3",
    "--expt-relaxed-constexpr",
    "-rdc=false",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "cetasim_gpu.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cmds, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
        objs.append(obj)
    # the translation units compile independently: one nvcc per source at once
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs,
           "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


CLI = os.path.join(HERE, "cetasim_mp")
HOST_SOURCES = ["mpbeam.cpp", "cbm_writer.cpp", "cetasim_mp.cpp"]


def build_host(force: bool = False, verbose: bool = False) -> str:
    """The C++ host layer (MPBeam-named wrapper) and the cetasim_mp driver,
    linked against the in-tree libcetagpu.so."""
    hdir = os.path.join(HERE, "host")
    deps = [os.path.join(hdir, s) for s in HOST_SOURCES + ["mpbeam.hpp", "cbm_writer.hpp"]] + [
        LIB, os.path.join(ROOT, "include", "cetasim_gpu.h")]
    if not force and not _stale(CLI, deps):
        return CLI
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-o", CLI + ".tmp",
           *[os.path.join(hdir, s) for s in HOST_SOURCES], "-L" + HERE, "-lcetagpu",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(CLI + ".tmp", CLI)
    return CLI


def build_oracle(verbose: bool = False) -> None:
    """Builds the CPU oracle (test infrastructure).  With the CETASim source
    tree named by the environment variable CETASIM_REFERENCE, also builds
    the reference's own sources into oracle/_ref (its compiled w(z), and its
    multi-particle path with the harness: see oracle/Makefile); without it,
    oracle/_ref keeps whatever an earlier build left there."""
    odir = os.path.join(ROOT, "oracle")
    subprocess.run(["make", "-s", "-C", odir, "CC=gcc", "CXX=g++"], check=True,
                   stdout=None if verbose else subprocess.DEVNULL)
    ref_src = os.environ.get("CETASIM_REFERENCE")
    if not ref_src:
        if verbose:
            print("CETASIM_REFERENCE not set: oracle/_ref not rebuilt", flush=True)
        return
    if not os.path.exists(os.path.join(ref_src, "src", "MPBeam.cpp")):
        raise RuntimeError(f"CETASIM_REFERENCE={ref_src} holds no src/MPBeam.cpp")
    subprocess.run(["make", "-s", f"-j{os.cpu_count() or 1}", "-C", odir, "ref", f"REF={ref_src}",
                    "CC=gcc", "CXX=g++"], check=True,
                   stdout=None if verbose else subprocess.DEVNULL,
                   stderr=None if verbose else subprocess.DEVNULL)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="-v" in sys.argv)
    build_host(force="--force" in sys.argv, verbose=True)
    build_oracle(verbose=True)
    print(LIB)
