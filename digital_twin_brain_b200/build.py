"""Build of libdtb.so (CUDA kernels + C ABI) for sm_100a, in-tree.

``python -m digital_twin_brain_b200.build`` or :func:`build` compiles
``csrc/dtb_api.cu`` and ``csrc/dtb_io.cpp`` with nvcc into
``digital_twin_brain_b200/libdtb.so``.  Cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libdtb.so")
# bench.py's measurement helper (float2 atomic rate), kept out of libdtb.so
PROBE_LIB = os.path.join(PKG, "libdtb_bench_probe.so")
PROBE_SOURCES = ["bench_probe.cu"]

SOURCES = ["dtb_api.cu", "dtb_prealloc.cu", "dtb_mlp.cu", "dtb_io.cpp"]
HEADERS = ["dtb_device.cuh", "dtb_kernels.cuh", "dtb_io.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # the neuron update restates torch's float32 operation order: never fuse a*b+c
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdtb.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "dtb.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    build_probe(force)
    if not force and not _stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES] + ["-lz"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_probe(force: bool = False) -> str:
    """libdtb_bench_probe.so: the float2 atomic-rate probe bench.py reports beside the push scatter."""
    srcs = [os.path.join(CSRC, f) for f in PROBE_SOURCES]
    if not force and os.path.exists(PROBE_LIB) and all(os.path.getmtime(f) <= os.path.getmtime(PROBE_LIB)
                                                        for f in srcs + [__file__]):
        return PROBE_LIB
    subprocess.check_call([nvcc()] + NVCC_FLAGS + ["-o", PROBE_LIB + ".tmp"] + srcs)
    os.replace(PROBE_LIB + ".tmp", PROBE_LIB)
    return PROBE_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
