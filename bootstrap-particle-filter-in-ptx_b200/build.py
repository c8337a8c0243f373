"""Build step of the CUDA library libgpubpf.so (sm_100a only).

Run as ``python bootstrap-particle-filter-in-ptx_b200/build.py`` or through
``__graft_entry__.build()``. The library is written in-tree next to the
Python binding (``gpubpf/libgpubpf.so``) so it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "gpubpf", "libgpubpf.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["bpf_alloc.cu", "bpf_plain.cu", "bpf_api.cu", "bpf_static.cu", "bpf_batch.cu", "bpf_batch_api.cu", "bpf_grad.cu",
           "bpf_grad_api.cu", "bpf_imm.cu", "bpf_smc2.cu", "bpf_apf.cu"]
HEADERS = ["bpf_alloc.cuh", "bpf_common.cuh", "bpf_plain.cuh", "bpf_block.cuh", "bpf_batch.cuh", "bpf_grad.cuh",
           "bpf_batch_internal.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xcompiler", "-fvisibility=default",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


OBJ_DIR = os.path.join(HERE, "_build")


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile libgpubpf.so if any source is newer than it; return its path. The sources are
    compiled to objects in parallel (one nvcc per source) and linked into the shared library."""
    from concurrent.futures import ThreadPoolExecutor
    headers = [os.path.join(CSRC, f) for f in HEADERS] + [os.path.join(INCLUDE, "gpu_bpf.h")]
    deps = [os.path.join(CSRC, f) for f in SOURCES] + headers
    if not force and not _stale(OUT, deps):
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        if force or _stale(obj, [os.path.join(CSRC, src)] + headers):
            cmd = [_nvcc(), *compile_flags, "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            os.replace(obj + ".tmp", obj)
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
