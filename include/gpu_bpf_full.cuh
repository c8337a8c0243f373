/*
 * gpu_bpf_full.cuh — source-compatibility name of include/gpu_bpf.h.
 *
 * The reference's PTX edition declares its API in gpu_bpf/gpu_bpf_full.cuh
 * (included by callers built with USE_PTX_FULL, e.g.
 * tests/bench_particle_scaling.cu:19-20). Every function that header declares
 * for the bootstrap filter, its online learning and the auxiliary particle
 * filter is declared in gpu_bpf.h under the same name and argument list.
 */
#ifndef GPU_BPF_FULL_CUH_COMPAT
#define GPU_BPF_FULL_CUH_COMPAT
#include "gpu_bpf.h"
#endif
