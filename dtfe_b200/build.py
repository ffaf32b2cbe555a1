"""Build recipes for the native libraries (in-tree, no JIT cache).

* ``libdtfe_host.so``  — host tessellator and sub-box planning (g++/OpenMP)
* ``libdtfe_gpu.so``   — CUDA kernels + C ABI of include/dtfe_gpu.h, sm_100a
* ``liboracle.so``     — the CPU oracle (test infrastructure, under oracle/)

Every library is written to a ``_build`` folder next to its sources so that it
travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dtfe_b200")
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
ORACLE = os.path.join(ROOT, "oracle")
ORACLE_BUILD = os.path.join(ORACLE, "_build")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["delaunay.cpp", "host_plan.cpp", "plan_build.cpp", "host_io.cpp"]
GPU_SOURCES = ["dtfe_core.cu", "deposit.cu", "adjoint.cu", "sph.cu", "method1.cu", "noalloc.cu",
               "delaunay.cu"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers(folder: str) -> list[str]:
    return [os.path.join(folder, f) for f in os.listdir(folder) if f.endswith((".h", ".cuh"))]


def build_host(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libdtfe_host.so")
    srcs = [os.path.join(CSRC, s) for s in HOST_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if force or _stale(out, srcs + _headers(CSRC) + _headers(INCLUDE)):
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
              "-I", INCLUDE, "-o", out] + srcs)
    return out


def build_gpu(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libdtfe_gpu.so")
    srcs = [os.path.join(CSRC, s) for s in GPU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if force or _stale(out, srcs + _headers(CSRC) + _headers(INCLUDE)):
        # -fmad=false: the interpolation arithmetic mirrors the reference's
        # separately rounded products (no FMA contraction).
        _run([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false",
                              "-Xcompiler", "-fPIC", "-shared", "-I", INCLUDE,
                              "-o", out] + srcs)
    return out


def build_oracle(force: bool = False) -> str:
    os.makedirs(ORACLE_BUILD, exist_ok=True)
    out = os.path.join(ORACLE_BUILD, "liboracle.so")
    srcs = [os.path.join(ORACLE, f) for f in sorted(os.listdir(ORACLE)) if f.endswith(".cpp")]
    if force or _stale(out, srcs + _headers(CSRC) + _headers(INCLUDE)):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
              "-I", INCLUDE, "-o", out] + srcs)
    return out


# the reference source tree (read only; the harness and the drop-in compile
# against it where it exists): DTFE_REFERENCE_TREE, else the default checkout
REFERENCE_TREE = os.environ.get("DTFE_REFERENCE_TREE", "/root/reference")


def build_ref() -> str | None:
    """The reference-code harness (oracle/_ref), only where the reference tree
    exists; elsewhere the prebuilt library, if any, is used as is."""
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        return None
    _run(["make", "-s", "-C", ORACLE, "ref", "refmain", "REF=" + REFERENCE_TREE])
    return os.path.join(ORACLE, "_ref", "libdtfe_ref.so")


SHIM = os.path.join(PKG, "shim")


def build_dropin(force: bool = False) -> str | None:
    """The DTFE() drop-in (dtfe_b200/shim/dtfe_drop_in.cpp -> libdtfe_dropin.so),
    compiled against the reference's own headers with the reference
    Makefile's default macros (3-D, velocity, one scalar).  Only where the
    reference tree exists; the boost headers its user_options.h includes come
    from the harness stand-ins here (a real build uses the caller's boost).
    Elsewhere the prebuilt library, if any, is used as is."""
    src_dir = os.path.join(REFERENCE_TREE, "src")
    if not os.path.isdir(src_dir):
        return None
    host, gpu = build_host(), build_gpu()
    out = os.path.join(BUILD, "libdtfe_dropin.so")
    src = os.path.join(SHIM, "dtfe_drop_in.cpp")
    if force or _stale(out, [src, host, gpu] + _headers(INCLUDE)):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-w",
              "-DNO_DIM=3", "-DVELOCITY", "-DSCALAR", "-DNO_SCALARS=1",
              "-I", INCLUDE, "-I", os.path.join(ORACLE, "refharness", "include"), "-I", src_dir,
              "-o", out, src, "-L", BUILD, "-ldtfe_host", "-ldtfe_gpu", "-Wl,-rpath,$ORIGIN"])
    return out


def build_dropin_driver() -> str | None:
    """Test driver of the drop-in (oracle/_ref/libdropin_driver.so): needs the
    reference tree, like the harness it links."""
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        return None
    _run(["make", "-s", "-C", ORACLE, "dropin", "REF=" + REFERENCE_TREE])
    return os.path.join(ORACLE, "_ref", "libdropin_driver.so")


def build_all(force: bool = False) -> None:
    build_host(force)
    build_gpu(force)
    build_oracle(force)
    build_ref()
    if build_dropin(force):
        build_dropin_driver()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built:", BUILD, ORACLE_BUILD)
