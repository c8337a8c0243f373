"""ctypes binding of libgpubpf.so (declarations in include/gpu_bpf.h).

The library is loaded from this directory only. There is no fallback: if the
shared object is missing or fails to load, importing a compute entry point
raises, so a GPU run can never silently execute anything but the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgpubpf.so")

BPF_OK = 0
BPF_ERR_ARG = 1
BPF_ERR_CUDA = 2
BPF_ERR_ALLOC = 3
BPF_ERR_UNSUPPORTED = 4
BPF_ERR_STATE = 5
BPF_ERR_DEGENERATE = 6
BPF_ERR_NODEVICE = 7
BPF_STATIC_MAX_PARTICLES = 262144


class BpfResult(C.Structure):
    """gpu_bpf/gpu_bpf.cuh:21-24 layout."""
    _fields_ = [("h_mean", C.c_float), ("log_lik", C.c_float)]


class BpfTickRecord(C.Structure):
    _fields_ = [
        ("dloglik", C.c_double),
        ("loglik_ref", C.c_double),
        ("loglik_total", C.c_double),
        ("h_mean", C.c_float),
        ("ess", C.c_float),
        ("resampled", C.c_int32),
        ("tick", C.c_int32),
    ]


class GpuBpfState(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int),
        ("rho", C.c_float), ("sigma_z", C.c_float), ("mu", C.c_float),
        ("nu_state", C.c_float), ("nu_obs", C.c_float),
        ("silverman_shrink", C.c_float),
        ("ess_threshold", C.c_float),
        ("did_resample", C.c_int),
        ("resample_count", C.c_int),
        ("timestep", C.c_int),
        ("last_h_est", C.c_float),
        ("stream", C.c_void_p),
        ("impl", C.c_void_p),
    ]


class BpfBatchFilter(C.Structure):
    _fields_ = [("mu", C.c_float), ("rho", C.c_float), ("sigma_z", C.c_float), ("nu_obs", C.c_float),
                ("n_particles", C.c_int), ("seed", C.c_int), ("nu_state", C.c_float)]


class ImmModelParams(C.Structure):
    _fields_ = [("rho", C.c_float), ("sigma_z", C.c_float), ("mu", C.c_float), ("nu_state", C.c_float),
                ("nu_obs", C.c_float)]


class ImmResult(C.Structure):
    _fields_ = [("h_mean", C.c_float), ("vol", C.c_float), ("log_lik", C.c_float), ("best_model", C.c_int),
                ("best_prob", C.c_float)]


class GpuImmState(C.Structure):
    _fields_ = [("filters", C.c_void_p), ("n_models", C.c_int), ("n_particles_per_model", C.c_int),
                ("log_pi", C.POINTER(C.c_double)), ("log_pi_pred", C.POINTER(C.c_double)),
                ("log_T", C.POINTER(C.c_double)), ("timestep", C.c_int), ("impl", C.c_void_p)]


class BpfSmc2Prior(C.Structure):
    _fields_ = [("mu_mean", C.c_float), ("mu_sd", C.c_float), ("rho_lo", C.c_float), ("rho_hi", C.c_float),
                ("sigma_lo", C.c_float), ("sigma_hi", C.c_float)]


class GpuApfState(C.Structure):
    _fields_ = [("n_particles", C.c_int),
                ("rho", C.c_float), ("sigma_z", C.c_float), ("mu", C.c_float),
                ("nu_state", C.c_float), ("nu_obs", C.c_float),
                ("timestep", C.c_int), ("stream", C.c_void_p), ("impl", C.c_void_p)]


P_STATE = C.POINTER(GpuBpfState)
P_APF = C.POINTER(GpuApfState)
P_IMM = C.POINTER(GpuImmState)
_f = C.c_float
_i = C.c_int
_d = C.c_double
_vp = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    # reference API (gpu_bpf/gpu_bpf.cuh:56-85, gpu_bpf_full.cuh:197-230)
    "gpu_bpf_create": (P_STATE, [_i, _f, _f, _f, _f, _f, _i]),
    "gpu_bpf_destroy": (None, [P_STATE]),
    "gpu_bpf_step": (BpfResult, [P_STATE, _f]),
    "gpu_bpf_step_async": (None, [P_STATE, _f]),
    "gpu_bpf_get_result": (BpfResult, [P_STATE]),
    "gpu_bpf_run_rmse": (_d, [C.POINTER(_d), C.POINTER(_d), _i, _i, _f, _f, _f, _f, _f, _i]),
    "gpu_bpf_set_bands": (None, [_i, _i, C.POINTER(_f), C.POINTER(_f)]),
    "gpu_bpf_set_adaptive_bands": (None, [_i, C.POINTER(_f), C.POINTER(_f), _i, C.POINTER(_f), C.POINTER(_f), _i,
                                          C.POINTER(_f), C.POINTER(_f), _i, _f, _f]),
    "gpu_bpf_set_ess_threshold": (None, [P_STATE, _f]),
    "gpu_bpf_get_resample_count": (_i, [P_STATE]),
    "gpu_bpf_get_mu": (_f, [P_STATE]),
    "gpu_bpf_get_rho": (_f, [P_STATE]),
    "gpu_bpf_set_mu": (None, [P_STATE, _f]),
    "gpu_bpf_set_rho": (None, [P_STATE, _f]),
    "gpu_bpf_enable_mu_learning": (None, [P_STATE, _i, _i, _f, _f, _f]),
    "gpu_bpf_disable_mu_learning": (None, [P_STATE]),
    "gpu_bpf_enable_rho_learning": (None, [P_STATE, _i]),
    # additions
    "gpu_bpf_last_error": (_i, []),
    "gpu_bpf_error_string": (C.c_char_p, [_i]),
    "gpu_bpf_step_many": (_i, [P_STATE, C.POINTER(_f), _i, C.POINTER(BpfResult), C.POINTER(BpfTickRecord)]),
    "gpu_bpf_step_many_device": (_i, [P_STATE, _vp, _i, _vp]),
    "gpu_bpf_reset": (_i, [P_STATE, _i]),
    "gpu_bpf_get_record": (_i, [P_STATE, C.POINTER(BpfTickRecord)]),
    "gpu_bpf_get_ess": (_f, [P_STATE]),
    "gpu_bpf_get_loglik_total": (_d, [P_STATE]),
    "gpu_bpf_set_loglik_semantics": (_i, [P_STATE, _i]),
    "gpu_bpf_get_particles": (_i, [P_STATE, C.POINTER(_f)]),
    "gpu_bpf_record_ancestors": (_i, [P_STATE, _i]),
    "gpu_bpf_get_ancestors": (_i, [P_STATE, C.POINTER(C.c_int32)]),
    "gpu_bpf_get_resample_inputs": (_i, [P_STATE, C.POINTER(_f), C.POINTER(C.c_int32), C.POINTER(C.c_uint32)]),
    "gpu_bpf_profile": (_i, [P_STATE, _i]),
    "gpu_bpf_set_fused_small": (_i, [P_STATE, _i]),
    "gpu_bpf_checkpoint_bytes": (C.c_size_t, [P_STATE]),
    "gpu_bpf_save": (_i, [P_STATE, _vp, C.c_size_t]),
    "gpu_bpf_load": (_i, [P_STATE, _vp, C.c_size_t]),
    "gpu_bpf_profile_read": (_i, [P_STATE, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d), C.POINTER(_i),
                                  C.POINTER(_i)]),
    "gpu_bpf_launch_count": (C.c_longlong, []),
    "gpu_bpf_debug_fail_alloc": (_i, [C.c_longlong]),
    "gpu_bpf_debug_alloc_count": (C.c_longlong, []),
    "gpu_bpf_debug_live_allocs": (C.c_longlong, []),
    "gpu_bpf_get_learning_sums": (_i, [P_STATE, C.POINTER(_d), C.POINTER(_i)]),
    "gpu_bpf_run_static": (_i, [_i, _f, _f, _f, _f, _i, _f, _vp, _i, _vp, _vp]),
    # batched filters
    "gpu_bpf_batch_create": (_vp, [C.POINTER(BpfBatchFilter), _i, _f]),
    "gpu_bpf_batch_destroy": (None, [_vp]),
    "gpu_bpf_batch_stream": (_vp, [_vp]),
    "gpu_bpf_batch_size_class": (_i, [_i]),
    "gpu_bpf_batch_set_threads": (_i, [_vp, _i, _i]),
    "gpu_bpf_batch_get_threads": (_i, [_vp, _i]),
    "gpu_bpf_batch_autotune": (_i, [_vp, C.POINTER(_f), _i, C.c_char_p]),
    "gpu_bpf_batch_run": (_i, [_vp, C.POINTER(_f), _i, C.POINTER(_d), C.POINTER(_f)]),
    "gpu_bpf_batch_run_device": (_i, [_vp, _vp, _i, _vp, _vp, _vp]),
    "gpu_bpf_batch_run_debug": (_i, [_vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "gpu_bpf_batch_resample_counts": (_i, [_vp, C.POINTER(_i), C.POINTER(_f)]),
    "gpu_bpf_batch_grad_run": (_i, [_vp, _vp, _i, _vp, _vp]),
    "gpu_bpf_batch_step_device": (_i, [_vp, _vp, _i, _vp, _vp]),
    "gpu_bpf_batch_reset": (_i, [_vp]),
    "gpu_bpf_batch_set_filters": (_i, [_vp, C.POINTER(BpfBatchFilter)]),
    "gpu_bpf_batch_tick": (_i, [_vp]),
    "gpu_bpf_batch_loglik_device": (_vp, [_vp]),
    "gpu_bpf_batch_grad_tape_bytes": (C.c_size_t, [_vp, _i]),
    "gpu_bpf_batch_run_correlated": (_i, [_vp, _vp, _i, _vp, _vp, _f, _vp, _vp, _vp]),
    "gpu_bpf_batch_noise_offset": (C.c_longlong, [_vp, _i, _i]),
    # APF (gpu_bpf/gpu_bpf.cuh:114-126)
    "gpu_apf_create": (P_APF, [_i, _f, _f, _f, _f, _f, _i]),
    "gpu_apf_destroy": (None, [P_APF]),
    "gpu_apf_step": (BpfResult, [P_APF, _f]),
    "gpu_apf_run_rmse": (_d, [C.POINTER(_d), C.POINTER(_d), _i, _i, _f, _f, _f, _f, _f, _i]),
    "gpu_apf_step_many": (_i, [P_APF, C.POINTER(_f), _i, C.POINTER(BpfResult), C.POINTER(BpfTickRecord)]),
    "gpu_apf_get_record": (_i, [P_APF, C.POINTER(BpfTickRecord)]),
    "gpu_apf_get_loglik_total": (_d, [P_APF]),
    "gpu_apf_get_particles": (_i, [P_APF, C.POINTER(_f)]),
    "gpu_apf_record_ancestors": (_i, [P_APF, _i]),
    "gpu_apf_get_ancestors": (_i, [P_APF, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    # IMM (gpu_bpf/gpu_bpf.cuh:131-164)
    "gpu_imm_create": (P_IMM, [C.POINTER(ImmModelParams), _i, _i, C.POINTER(_f), _i]),
    "gpu_imm_step": (ImmResult, [P_IMM, _f]),
    "gpu_imm_get_prob": (_f, [P_IMM, _i]),
    "gpu_imm_get_probs": (None, [P_IMM, C.POINTER(_f)]),
    "gpu_imm_destroy": (None, [P_IMM]),
    "gpu_imm_build_grid": (C.POINTER(ImmModelParams), [C.POINTER(_f), _i, C.POINTER(_f), _i, C.POINTER(_f), _i,
                                                        _f, _f, C.POINTER(_i)]),
    # SMC^2
    "gpu_bpf_smc2_create": (_vp, [_i, _i, _i, C.POINTER(BpfSmc2Prior), C.c_ulonglong]),
    "gpu_bpf_smc2_destroy": (None, [_vp]),
    "gpu_bpf_smc2_set_moves": (_i, [_vp, _i, _f, _f]),
    "gpu_bpf_smc2_update": (_f, [_vp, _f]),
    "gpu_bpf_smc2_get_outer_ess": (_f, [_vp]),
    "gpu_bpf_smc2_get_theta": (_i, [_vp, C.POINTER(_f), C.POINTER(_f)]),
    "gpu_bpf_smc2_get_particles": (_i, [_vp, _vp, _vp, _vp]),
    "gpu_bpf_smc2_stats": (_i, [_vp, C.POINTER(_i), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "gpu_bpf_smc2_set_cpmmh_rho": (_i, [_vp, _f]),
    "gpu_bpf_smc2_get_last_move": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "gpu_bpf_smc2_get_last_update": (_i, [_vp, _vp, _vp, _vp]),
    "gpu_bpf_smc2_get_noise": (_i, [_vp, _i, _i, _vp]),
    # gradient
    "gpu_bpf_grad_create": (_vp, [_i, _i, _i]),
    "gpu_bpf_grad_destroy": (None, [_vp]),
    "gpu_bpf_grad_tape_bytes": (C.c_size_t, [_i, _i, _i]),
    "gpu_bpf_grad_stream": (_vp, [_vp]),
    "gpu_bpf_grad_checkpoint_every": (_i, [_vp]),
    "gpu_bpf_grad_forward": (_i, [_vp, _f, _f, _f, _f, _f, _i, _f, _vp, _i, _vp]),
    "gpu_bpf_grad_backward": (_i, [_vp, _vp]),
    "gpu_bpf_grad_replay": (_i, [_vp, _d, _d, _d, _vp, _vp]),
    "gpu_bpf_grad_get_records": (_i, [_vp, C.POINTER(BpfTickRecord), _i]),
    "gpu_bpf_grad_get_children": (_i, [_vp, _i, C.POINTER(C.c_int32)]),
    "gpu_bpf_debug_pcg32": (_i, [_i, _i, _i, C.POINTER(C.c_uint32)]),
    "gpu_bpf_debug_normals": (_i, [_i, _i, _i, C.POINTER(_f)]),
}

_LIB = None


def load() -> C.CDLL:
    """Load libgpubpf.so and declare every exported signature (raises if absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libgpubpf.so not found at {LIB_PATH}; build it with "
            "`python bootstrap-particle-filter-in-ptx_b200/build.py`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class BpfError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        lib = load()
        msg = lib.gpu_bpf_error_string(code).decode()
        super().__init__(f"{where}: BPF error {code} ({msg})" if where else f"BPF error {code} ({msg})")
        self.code = code


def check(rc: int, where: str = "") -> None:
    if rc != BPF_OK:
        raise BpfError(rc, where)
