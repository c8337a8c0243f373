/*
 * gpu_bpf.cuh — source-compatibility name of include/gpu_bpf.h.
 *
 * The reference's callers include the CUDA-C edition's header by this name
 * (gpu_bpf/gpu_bpf.cuh, e.g. tests/test_cond_resample.cu:19,
 * tests/bench_particle_scaling.cu:22). Putting this directory on the include
 * path in place of the reference's gpu_bpf/ lets such a caller build against
 * libgpubpf.so with no edit to its source.
 */
#ifndef GPU_BPF_CUH_COMPAT
#define GPU_BPF_CUH_COMPAT
#include "gpu_bpf.h"
#endif
