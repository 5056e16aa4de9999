"""Builds the engine's native libraries in-tree (they travel with the source tree to the GPU host).

* ``monoprop_b200/libmpx.so`` -- the CUDA engine behind the C ABI of ``include/mpx.h``, compiled for
  sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
* ``monoprop_b200/_core*.so`` -- the pybind11 module exposing the reference's per-tier engine classes
  (``MonomialPropagator032`` ...) over that C ABI.

Run ``python -m monoprop_b200.build`` (or ``__graft_entry__.build()``). nvcc cross-compiles without a GPU.
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmpx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(exts: tuple[str, ...]) -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(exts))


def build_engine(force: bool = False, verbose: bool = False) -> str:
    cu = [os.path.join(CSRC, "mpx_engine.cu"), os.path.join(CSRC, "mpx_noalloc.cu"), os.path.join(CSRC, "mpx_batch.cu")]
    deps = _sources((".cu", ".cuh", ".h")) + [os.path.join(ROOT, "include", "mpx.h")]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "-shared", "-I", os.path.join(ROOT, "include"), *cu, "-o", LIB,
               "-lcudart"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
    return LIB


def build_core(force: bool = False) -> str:
    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = os.path.join(PKG, "_core" + suffix)
    src = os.path.join(CSRC, "core_bindings.cpp")
    if force or _stale(target, [src, os.path.join(ROOT, "include", "mpx.h"), LIB]):
        inc = sysconfig.get_paths()["include"]
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I", inc,
               "-I", pybind11.get_include(), "-I", os.path.join(ROOT, "include"), src, "-o", target,
               "-L", PKG, "-lmpx", "-Wl,-rpath,$ORIGIN"]
        subprocess.check_call(cmd)
    return target


def build(force: bool = False, verbose: bool = False) -> None:
    build_engine(force=force, verbose=verbose)
    if os.path.exists(os.path.join(CSRC, "core_bindings.cpp")):
        build_core(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
