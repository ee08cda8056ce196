"""Builds the in-tree CUDA library for sm_100a with nvcc.

    python -m kraken_3_gpu_b200.build

Output: kraken_3_gpu_b200/libkraken_b200.so (kept out of git, shipped with the
tree), and the Node N-API addon's object napi/kraken_napi.o (compiled with
gcc against the Node-API declarations of napi/node_api_decls.h: a compile
check of the addon where no Node toolchain exists; node-gyp with
napi/binding.gyp builds the loadable addon).  -fmad=false keeps every f32 multiply and add separately rounded, as
the reference's per-op f32 semantics require; the kernels use explicit
non-fusing intrinsics as well.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libkraken_b200.so")
SOURCES = ["kr_world.cu", "kr_batch.cu", "kr_serve.cu", "kr_template.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    inc = os.path.join(os.path.dirname(HERE), "include")
    deps += [os.path.join(inc, f) for f in os.listdir(inc)]
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps):
            return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUT, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return OUT




NAPI_SRC = os.path.join(HERE, "napi", "kraken_napi.c")
NAPI_OBJ = os.path.join(HERE, "napi", "kraken_napi.o")


def build_napi_object() -> str:
    """Compile the N-API addon source to an object file (gcc, -Werror)."""
    inc = os.path.join(os.path.dirname(HERE), "include")
    cmd = [os.environ.get("CC", "gcc"), "-std=c11", "-O2", "-fPIC", "-Wall", "-Wextra", "-Werror",
           "-I", inc, "-I", os.path.dirname(NAPI_SRC), "-c", NAPI_SRC, "-o", NAPI_OBJ]
    subprocess.run(cmd, check=True)
    return NAPI_OBJ


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
    print(build_napi_object())
