"""Build the reference's own GPU filter into oracle/_ref/ (test infrastructure).

TEST INFRASTRUCTURE ONLY. The reference ships its plain filter as hand-written
PTX (ptx_assembly/bpf_kernels_full.ptx) loaded at run time by
gpu_bpf/gpu_bpf_ptx_full.cu. Two facts keep that module from loading unchanged
on a B200 with CUDA 12.9, and this recipe applies exactly those two edits to a
copy written under oracle/_ref/ (the reference tree is never modified):

  * the file carries UTF-8 bytes in comments (box-drawing characters near the
    kernel-14 banner), which ptxas rejects ("Unexpected non-ASCII character"):
    every byte above 0x7F is dropped; all of them sit in comments;
  * it declares `.target sm_120`, which the JIT refuses on sm_100: the line is
    rewritten to `.target sm_100a`.

The host driver (gpu_bpf_ptx_full.cu, with gpu_bpf_full.cuh) is compiled from
where it lies, together with oracle/ref_gpu_shim.cu (C-linkage wrappers), into
oracle/_ref/librefgpu.so. Nothing else of the reference is built; it needs the
CUDA driver library, cuRAND and thrust from the toolkit only.

A second library, oracle/_ref/librefcuda.so, is the reference's CUDA-C edition
(gpu_bpf/gpu_bpf.cu behind gpu_bpf/gpu_bpf.cuh, which holds the reference's
IMM) compiled from where it lies with oracle/ref_cuda_shim.cu. The two
editions export the same C++ names, so each gets its own library.

The output is git-ignored and travels with the repository snapshot to a GPU
machine; the reference tree itself is only read here, at build time.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "librefgpu.so")
PTX = os.path.join(OUT, "bpf_kernels_full.ptx")
SHIM = os.path.join(HERE, "ref_gpu_shim.cu")
LIB_C = os.path.join(OUT, "librefcuda.so")
SHIM_C = os.path.join(HERE, "ref_cuda_shim.cu")

# The reference tree: $BPF_REFERENCE_ROOT, else a checkout named `reference` beside this repository.
REF_ROOT = os.environ.get("BPF_REFERENCE_ROOT") or os.path.join(os.path.dirname(HERE), os.pardir, "reference")
REF_DRIVER = os.path.join(REF_ROOT, "gpu_bpf", "gpu_bpf_ptx_full.cu")
REF_PTX = os.path.join(REF_ROOT, "ptx_assembly", "bpf_kernels_full.ptx")
REF_CUDA = os.path.join(REF_ROOT, "gpu_bpf", "gpu_bpf.cu")


def available() -> bool:
    """True when the library and its PTX module are built."""
    return os.path.exists(LIB) and os.path.exists(PTX)


def available_cuda() -> bool:
    """True when the CUDA-C edition's library is built."""
    return os.path.exists(LIB_C)


def build_cuda(force: bool = False) -> str | None:
    """Build oracle/_ref/librefcuda.so (the CUDA-C edition) when the reference tree is present."""
    if not os.path.exists(REF_CUDA):
        return LIB_C if available_cuda() else None
    inputs = [REF_CUDA, SHIM_C, os.path.join(os.path.dirname(REF_CUDA), "gpu_bpf.cuh")]
    if not force and available_cuda() and os.path.getmtime(LIB_C) >= max(os.path.getmtime(p) for p in inputs):
        return LIB_C
    os.makedirs(OUT, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC", "-I", os.path.dirname(REF_CUDA),
           REF_CUDA, SHIM_C, "-o", LIB_C + ".tmp", "-lcurand"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    os.replace(LIB_C + ".tmp", LIB_C)
    return LIB_C


def _retarget(src: bytes) -> bytes:
    text = bytes(b for b in src if b < 0x80).decode("ascii")
    text, n = re.subn(r"^\.target\s+sm_\w+", ".target sm_100a", text, count=1, flags=re.M)
    if n != 1:
        raise RuntimeError("no .target line in the reference PTX")
    return text.encode("ascii")


def build(force: bool = False) -> str | None:
    """Build oracle/_ref/ when the reference tree is present; returns the library path or None."""
    if not (os.path.exists(REF_DRIVER) and os.path.exists(REF_PTX)):
        return LIB if available() else None
    inputs = [REF_DRIVER, REF_PTX, SHIM, os.path.join(os.path.dirname(REF_DRIVER), "gpu_bpf_full.cuh")]
    if not force and available() and os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in inputs):
        return LIB
    os.makedirs(OUT, exist_ok=True)
    with open(REF_PTX, "rb") as f:
        ptx = _retarget(f.read())
    with open(PTX + ".tmp", "wb") as f:
        f.write(ptx)
    os.replace(PTX + ".tmp", PTX)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC", "-I", os.path.dirname(REF_DRIVER),
           REF_DRIVER, SHIM, "-o", LIB + ".tmp", "-lcuda", "-lcurand", "-ldl"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv)
    print(path or "reference tree absent; oracle/_ref not built")
    print(build_cuda(force="--force" in sys.argv) or "reference tree absent; CUDA-C edition not built")
