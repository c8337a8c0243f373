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

The drop-in check (build_dropin) compiles some of the reference's own caller
programs (its tests and benchmarks that use the host API) from where they lie,
unchanged, against this repository's include/ directory (which answers to the
reference header names gpu_bpf.cuh and gpu_bpf_full.cuh) and links them to
libgpubpf.so, into oracle/_ref/dropin/. tests/test_gpu_dropin.py runs them.

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


REPO = os.path.dirname(HERE)
INCLUDE = os.path.join(REPO, "include")
PKG_LIB_DIR = os.path.join(REPO, "bootstrap-particle-filter-in-ptx_b200", "gpubpf")
DROPIN = os.path.join(OUT, "dropin")
# reference caller programs built unchanged against include/ + libgpubpf.so: (output name, source, defines)
DROPIN_PROGRAMS = [
    ("bench_particle_scaling", os.path.join("tests", "bench_particle_scaling.cu"), []),
    ("bench_particle_scaling_ptx_full", os.path.join("tests", "bench_particle_scaling.cu"), ["-DUSE_PTX_FULL=1"]),
    ("test_cond_resample", os.path.join("tests", "test_cond_resample.cu"), []),
    ("test_bpf_matched_dgp", os.path.join("tests", "test_bpf_matched_dgp.cu"), []),
    ("test_mu_learning", os.path.join("smc2", "test_mu_learning.cu"), []),
    ("bench_grad_overhead", os.path.join("tests", "bench_grad_overhead.cu"), []),
]


def dropin_path(name: str) -> str:
    return os.path.join(DROPIN, name)


def build_dropin(force: bool = False) -> list:
    """Compile the reference caller programs of DROPIN_PROGRAMS, unmodified, against include/ and
    libgpubpf.so (run-time search path relative to the executable). Returns the names built or up
    to date; nothing when the reference tree is absent."""
    lib = os.path.join(PKG_LIB_DIR, "libgpubpf.so")
    if not os.path.exists(lib):
        return []
    headers = [os.path.join(INCLUDE, h) for h in ("gpu_bpf.h", "gpu_bpf.cuh", "gpu_bpf_full.cuh")]
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    rpath = "$ORIGIN/" + os.path.relpath(PKG_LIB_DIR, DROPIN)
    done = []
    for name, rel, defs in DROPIN_PROGRAMS:
        src = os.path.join(REF_ROOT, rel)
        out = dropin_path(name)
        if not os.path.exists(src):
            if os.path.exists(out):
                done.append(name)
            continue
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(p) for p in [src] + headers):
            done.append(name)
            continue
        os.makedirs(DROPIN, exist_ok=True)
        cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", *defs, "-I", INCLUDE, src,
               "-o", out + ".tmp", "-L", PKG_LIB_DIR, "-lgpubpf", "-Xlinker", "-rpath", "-Xlinker", rpath]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        os.replace(out + ".tmp", out)
        done.append(name)
    return done


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
    print("drop-in programs:", build_dropin(force="--force" in sys.argv))
