"""Builds libccb.so in-tree for sm_100a (B200) with nvcc.

    python -m cuda_graph_clustering_b200.build [--force] [--cc-gpu [REFERENCE_ROOT]]

Every CUDA source is compiled with ``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into an
object under ``cuda_graph_clustering_b200/_build`` and linked into
``cuda_graph_clustering_b200/libccb.so``.  Objects are rebuilt only when a source or header is newer.
With ``--cc-gpu`` it also links the drop-in ``cc_gpu`` binary (the reference's command line on libccb) from
the reference checkout given after the flag or in CCB_REFERENCE.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libccb.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I", os.path.join(REPO, "include"),
          "-I", CSRC, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if _stale(obj, [src] + _headers()):
        cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{proc.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in glob.glob(os.path.join(BUILD, "*.o")):
            os.remove(f)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(_compile, srcs))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{proc.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


CC_GPU = os.path.join(PKG, "cc_gpu")


def build_cc_gpu(reference: str | None = None, verbose: bool = False) -> str | None:
    """The drop-in cc_gpu binary: the reference's own command line (include/cc_cli.hpp) and host sources
    (src/cc_graph.cpp, src/cc_pbils_cpu.cpp), compiled where they lie, linked with cc_gpu_ccb.cpp (the
    reference's GPU entry points over libccb) and libccb.so.  `reference` is the reference checkout's root
    (default: the CCB_REFERENCE environment variable).  Returns the binary's path, or None when no checkout
    is given or it lacks those sources."""
    reference = reference or os.environ.get("CCB_REFERENCE")
    if not reference:
        return None
    inc = os.path.join(reference, "include")
    srcs = [os.path.join(reference, "src", f) for f in ("cc_graph.cpp", "cc_pbils_cpu.cpp")]
    if not all(os.path.exists(x) for x in [inc] + srcs):
        return None
    lib = build()
    deps = srcs + [os.path.join(PKG, "cc_gpu_ccb.cpp"), lib, os.path.join(REPO, "include", "ccb.h")]
    if _stale(CC_GPU, deps):
        cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-pthread", "-DCCB_CC_GPU_MAIN", "-I", inc,
               "-I", os.path.join(REPO, "include"), os.path.join(PKG, "cc_gpu_ccb.cpp")] + srcs + \
              ["-L", PKG, "-lccb", "-Wl,-rpath,$ORIGIN", "-o", CC_GPU]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"cc_gpu link failed:\n{proc.stderr}")
        if verbose:
            print("linked", CC_GPU)
    return CC_GPU


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    if "--cc-gpu" in sys.argv:  # python -m cuda_graph_clustering_b200.build --cc-gpu [REFERENCE_ROOT]
        at = sys.argv.index("--cc-gpu")
        print(build_cc_gpu(sys.argv[at + 1] if at + 1 < len(sys.argv) else None, verbose=True))
