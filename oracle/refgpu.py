"""ctypes face of the reference's own GPU filter built into oracle/_ref/ by oracle/build_ref.py.

TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle and the CUDA path
against the reference itself run on the same GPU, and by bench.py's reference
arm to time it. The product never imports it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import build_ref

_LIB = None


def available() -> bool:
    return build_ref.available()


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not build_ref.available():
            raise RuntimeError("oracle/_ref is not built (the reference tree was absent at build time)")
        L = C.CDLL(build_ref.LIB)
        vp, f32, i32, f64 = C.c_void_p, C.c_float, C.c_int, C.c_double
        L.refgpu_create.restype = vp
        L.refgpu_create.argtypes = [i32, f32, f32, f32, f32, f32, i32]
        L.refgpu_destroy.argtypes = [vp]
        L.refgpu_set_ess.argtypes = [vp, f32]
        L.refgpu_resample_count.restype = i32
        L.refgpu_resample_count.argtypes = [vp]
        L.refgpu_timestep.restype = i32
        L.refgpu_timestep.argtypes = [vp]
        L.refgpu_run.restype = i32
        L.refgpu_run.argtypes = [vp, vp, i32, vp, vp]
        L.refgpu_time_run.restype = f64
        L.refgpu_time_run.argtypes = [vp, vp, i32, vp]
        L.refgpu_enable_mu_learning.argtypes = [vp, i32, i32, f32, f32, f32]
        L.refgpu_enable_rho_learning.argtypes = [vp, i32]
        L.refgpu_get_mu.restype = f32
        L.refgpu_get_mu.argtypes = [vp]
        L.refgpu_get_rho.restype = f32
        L.refgpu_get_rho.argtypes = [vp]
        L.refgpu_time_steps.restype = f64
        L.refgpu_time_steps.argtypes = [vp, vp, i32, i32]
        L.refgpu_apf_create.restype = vp
        L.refgpu_apf_create.argtypes = [i32, f32, f32, f32, f32, f32, i32]
        L.refgpu_apf_destroy.argtypes = [vp]
        L.refgpu_apf_time.restype = f64
        L.refgpu_apf_time.argtypes = [vp, vp, i32]
        L.refgpu_apf_run.restype = i32
        L.refgpu_apf_run.argtypes = [vp, vp, i32, vp, vp]
        for name in ("refgpu_copy_rng", "refgpu_copy_h", "refgpu_copy_h2", "refgpu_copy_w"):
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [vp, vp, i32]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RefGpuFilter:
    """gpu_bpf_create / gpu_bpf_step / gpu_bpf_destroy of the reference's PTX edition."""

    def __init__(self, n, rho, sigma_z, mu, nu_state=0.0, nu_obs=0.0, seed=42, ess_threshold=0.5):
        self.L = lib()
        self.n = int(n)
        self.s = self.L.refgpu_create(self.n, rho, sigma_z, mu, nu_state, nu_obs, int(seed))
        if not self.s:
            raise RuntimeError("reference gpu_bpf_create failed")
        self.L.refgpu_set_ess(self.s, float(ess_threshold))

    def run(self, y):
        """One gpu_bpf_step per observation: (h_mean[T], log_lik[T]) as float32."""
        y = np.ascontiguousarray(y, dtype=np.float32)
        hm = np.zeros(y.shape[0], dtype=np.float32)
        ll = np.zeros(y.shape[0], dtype=np.float32)
        rc = self.L.refgpu_run(self.s, _p(y), int(y.shape[0]), _p(hm), _p(ll))
        if rc != 0:
            raise RuntimeError(f"reference tick loop failed (CUDA error {rc})")
        return hm, ll

    def time_run(self, y):
        """gpu_bpf_step_async over y, one result at the end: (milliseconds, h_mean, log_lik)."""
        y = np.ascontiguousarray(y, dtype=np.float32)
        last = np.zeros(2, dtype=np.float32)
        ms = self.L.refgpu_time_run(self.s, _p(y), int(y.shape[0]), _p(last))
        return ms, float(last[0]), float(last[1])

    def enable_mu_learning(self, mode=1, K=50, c=0.1, t0=10.0, gamma=0.667):
        self.L.refgpu_enable_mu_learning(self.s, int(mode), int(K), float(c), float(t0), float(gamma))

    def enable_rho_learning(self, enable=True):
        self.L.refgpu_enable_rho_learning(self.s, int(enable))

    def mu(self):
        return float(self.L.refgpu_get_mu(self.s))

    def rho_value(self):
        return float(self.L.refgpu_get_rho(self.s))

    def time_steps(self, y, warmup=100):
        """warmup untimed then len(y) timed ticks of gpu_bpf_step in a C loop: milliseconds."""
        y = np.ascontiguousarray(y, dtype=np.float32)
        return float(self.L.refgpu_time_steps(self.s, _p(y), int(y.shape[0]), int(warmup)))

    def _copy(self, name, dtype, count):
        out = np.zeros(count, dtype=dtype)
        rc = getattr(self.L, name)(self.s, _p(out), self.n)
        if rc != 0:
            raise RuntimeError(f"{name} failed (CUDA error {rc})")
        return out

    def rng(self):
        """PCG32 [state, inc] per particle, shape (N, 2) uint64."""
        return self._copy("refgpu_copy_rng", np.uint64, 2 * self.n).reshape(self.n, 2)

    def particles(self):
        return self._copy("refgpu_copy_h", np.float32, self.n)

    def pre_resample_particles(self):
        return self._copy("refgpu_copy_h2", np.float32, self.n)

    def weights(self):
        return self._copy("refgpu_copy_w", np.float32, self.n)

    @property
    def resample_count(self):
        return self.L.refgpu_resample_count(self.s)

    @property
    def timestep(self):
        return self.L.refgpu_timestep(self.s)

    def close(self):
        if self.s:
            self.L.refgpu_destroy(self.s)
            self.s = None


def apf_run(n, rho, sigma_z, mu, y, nu_state=0.0, nu_obs=0.0, seed=42):
    """The reference's gpu_apf_create / gpu_apf_step loop: (h_mean[T], log_lik[T]) float32."""
    L = lib()
    s = L.refgpu_apf_create(int(n), rho, sigma_z, mu, nu_state, nu_obs, int(seed))
    if not s:
        raise RuntimeError("reference gpu_apf_create failed")
    try:
        y = np.ascontiguousarray(y, dtype=np.float32)
        hm = np.zeros(y.shape[0], dtype=np.float32)
        ll = np.zeros(y.shape[0], dtype=np.float32)
        rc = L.refgpu_apf_run(s, _p(y), int(y.shape[0]), _p(hm), _p(ll))
        if rc != 0:
            raise RuntimeError(f"reference APF loop failed (CUDA error {rc})")
        return hm, ll
    finally:
        L.refgpu_apf_destroy(s)


def apf_time(n, rho, sigma_z, mu, y, warmup=64, seed=42):
    """Milliseconds per tick of the reference's APF over y[warmup:], after `warmup` untimed ticks."""
    L = lib()
    s = L.refgpu_apf_create(int(n), rho, sigma_z, mu, 0.0, 0.0, int(seed))
    if not s:
        raise RuntimeError("reference gpu_apf_create failed")
    try:
        y = np.ascontiguousarray(y, dtype=np.float32)
        L.refgpu_apf_time(s, _p(y[:warmup]), int(warmup))
        rest = np.ascontiguousarray(y[warmup:])
        ms = L.refgpu_apf_time(s, _p(rest), int(rest.shape[0]))
        return ms / rest.shape[0]
    finally:
        L.refgpu_apf_destroy(s)


# ---------------------------------------------------------------------------
# The reference's CUDA-C edition (oracle/_ref/librefcuda.so): plain filter and IMM
# ---------------------------------------------------------------------------
_LIBC = None


def available_cuda() -> bool:
    return build_ref.available_cuda()


def lib_cuda() -> C.CDLL:
    global _LIBC
    if _LIBC is None:
        if not build_ref.available_cuda():
            raise RuntimeError("oracle/_ref/librefcuda.so is not built")
        L = C.CDLL(build_ref.LIB_C)
        vp, f32, i32 = C.c_void_p, C.c_float, C.c_int
        L.refc_create.restype = vp
        L.refc_create.argtypes = [i32, f32, f32, f32, f32, f32, i32, f32, f32]
        L.refc_destroy.argtypes = [vp]
        L.refc_resample_count.restype = i32
        L.refc_resample_count.argtypes = [vp]
        L.refc_run.restype = i32
        L.refc_run.argtypes = [vp, vp, i32, vp, vp]
        L.refc_imm_create.restype = vp
        L.refc_imm_create.argtypes = [vp, i32, i32, vp, i32, f32, f32]
        L.refc_imm_destroy.argtypes = [vp]
        L.refc_imm_run.restype = i32
        L.refc_imm_run.argtypes = [vp, vp, i32, vp, vp, vp, vp]
        _LIBC = L
    return _LIBC


def cuda_run(n, rho, sigma_z, mu, y, nu_state=0.0, nu_obs=0.0, seed=42, ess_threshold=0.5, silverman=0.0):
    """The CUDA-C edition's plain filter over y (gpu_bpf_step per tick): (h_mean[T], log_lik[T],
    resample count)."""
    L = lib_cuda()
    y = np.ascontiguousarray(y, dtype=np.float32)
    s = L.refc_create(int(n), rho, sigma_z, mu, nu_state, nu_obs, int(seed), silverman, ess_threshold)
    if not s:
        raise RuntimeError("CUDA-C edition gpu_bpf_create failed")
    hm = np.zeros(y.shape[0], dtype=np.float32)
    ll = np.zeros(y.shape[0], dtype=np.float32)
    rc = L.refc_run(s, _p(y), int(y.shape[0]), _p(hm), _p(ll))
    cnt = L.refc_resample_count(s)
    L.refc_destroy(s)
    if rc != 0:
        raise RuntimeError(f"CUDA-C edition tick loop failed (CUDA error {rc})")
    return hm, ll, cnt


def cuda_imm_run(models, n, y, transition=None, seed=42, silverman=0.0, ess_threshold=0.5):
    """The CUDA-C edition's IMM over y: (h_mean[T], log_lik[T], best_model[T], final probs[K]).
    ess_threshold applies to every model's filter (its default is 0.5)."""
    L = lib_cuda()
    K = len(models)
    m = np.array([[d["rho"], d["sigma_z"], d["mu"], d.get("nu_state", 0.0), d.get("nu_obs", 0.0)] for d in models],
                 dtype=np.float32).ravel()
    tm = None if transition is None else np.ascontiguousarray(transition, dtype=np.float32)
    s = L.refc_imm_create(_p(m), K, int(n), _p(tm) if tm is not None else None, int(seed), silverman,
                          ess_threshold)
    if not s:
        raise RuntimeError("CUDA-C edition gpu_imm_create failed")
    y = np.ascontiguousarray(y, dtype=np.float32)
    hm = np.zeros(y.shape[0], dtype=np.float32)
    ll = np.zeros(y.shape[0], dtype=np.float32)
    best = np.zeros(y.shape[0], dtype=np.int32)
    pr = np.zeros(K, dtype=np.float32)
    rc = L.refc_imm_run(s, _p(y), int(y.shape[0]), _p(hm), _p(ll), _p(best), _p(pr))
    L.refc_imm_destroy(s)
    if rc != 0:
        raise RuntimeError(f"CUDA-C edition IMM failed (CUDA error {rc})")
    return hm, ll, best, pr
