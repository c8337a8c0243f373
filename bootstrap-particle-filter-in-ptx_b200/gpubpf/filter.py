"""Python mirror of the reference host API (gpu_bpf/gpu_bpf.cuh:56-85).

``GpuBpf`` wraps one ``GpuBpfState*`` of libgpubpf.so. Method names and
argument meaning follow the C functions (``step``, ``step_async``,
``get_result``, ``set_ess_threshold``, ``get_resample_count`` ...); errors
raise ``BpfError`` with the library's status code instead of the reference's
silent failure.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

from . import _lib
from ._lib import BpfError, BpfResult, BpfTickRecord, check


class GpuBpf:
    def __init__(self, n_particles: int, rho: float, sigma_z: float, mu: float,
                 nu_state: float = 0.0, nu_obs: float = 0.0, seed: int = 42,
                 ess_threshold: Optional[float] = None):
        self._lib = _lib.load()
        ptr = self._lib.gpu_bpf_create(int(n_particles), rho, sigma_z, mu, nu_state, nu_obs, int(seed))
        if not ptr:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_create")
        self._s = ptr
        self.n_particles = int(n_particles)
        if ess_threshold is not None:
            self.set_ess_threshold(ess_threshold)

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_s", None):
            self._lib.gpu_bpf_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def state(self) -> _lib.GpuBpfState:
        return self._s.contents

    # -- online mu / rho learning (gpu_bpf/gpu_bpf_full.cuh:176-204) --------
    def enable_mu_learning(self, mode: int = 1, K: int = 50, c: float = 0.1, t0: float = 10.0,
                           gamma: float = 0.667) -> None:
        self._lib.gpu_bpf_enable_mu_learning(self._s, int(mode), int(K), float(c), float(t0), float(gamma))

    def disable_mu_learning(self) -> None:
        self._lib.gpu_bpf_disable_mu_learning(self._s)

    def enable_rho_learning(self, enable: bool = True) -> None:
        self._lib.gpu_bpf_enable_rho_learning(self._s, int(bool(enable)))

    def learning_sums(self):
        arr = (C.c_double * 4)()
        n = C.c_int(0)
        check(self._lib.gpu_bpf_get_learning_sums(self._s, arr, C.byref(n)), "gpu_bpf_get_learning_sums")
        return list(arr), n.value

    # -- reference API ----------------------------------------------------
    def step(self, y_t: float) -> BpfResult:
        r = self._lib.gpu_bpf_step(self._s, float(y_t))
        if math.isnan(r.h_mean):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_step")
        return r

    def step_async(self, y_t: float) -> None:
        self._lib.gpu_bpf_step_async(self._s, float(y_t))

    def get_result(self) -> BpfResult:
        r = self._lib.gpu_bpf_get_result(self._s)
        if math.isnan(r.h_mean):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_get_result")
        return r

    def set_ess_threshold(self, thr: float) -> None:
        self._lib.gpu_bpf_set_ess_threshold(self._s, float(thr))

    def get_resample_count(self) -> int:
        n = self._lib.gpu_bpf_get_resample_count(self._s)
        if n < 0:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_get_resample_count")
        return n

    def get_mu(self) -> float:
        return self._lib.gpu_bpf_get_mu(self._s)

    def get_rho(self) -> float:
        return self._lib.gpu_bpf_get_rho(self._s)

    def set_mu(self, mu: float) -> None:
        self._lib.gpu_bpf_set_mu(self._s, float(mu))

    def set_rho(self, rho: float) -> None:
        self._lib.gpu_bpf_set_rho(self._s, float(rho))

    # -- additions --------------------------------------------------------
    def step_many(self, y: Sequence[float], records: bool = False):
        """Run len(y) ticks; returns a list of BpfResult (or BpfTickRecord)."""
        n = len(y)
        ya = (C.c_float * n)(*[float(v) for v in y])
        out = (BpfResult * n)()
        rec = (BpfTickRecord * n)() if records else None
        check(self._lib.gpu_bpf_step_many(self._s, ya, n, out, rec), "gpu_bpf_step_many")
        return list(rec) if records else list(out)

    def reset(self, seed: int) -> None:
        check(self._lib.gpu_bpf_reset(self._s, int(seed)), "gpu_bpf_reset")

    def step_many_device(self, y_dev_ptr: int, n_ticks: int, rec_dev_ptr: int) -> None:
        """Enqueue n_ticks ticks on device buffers (y f32[n], records 40 B x n)."""
        check(self._lib.gpu_bpf_step_many_device(self._s, C.c_void_p(y_dev_ptr), int(n_ticks),
                                                 C.c_void_p(rec_dev_ptr)), "gpu_bpf_step_many_device")

    def get_record(self) -> BpfTickRecord:
        r = BpfTickRecord()
        check(self._lib.gpu_bpf_get_record(self._s, C.byref(r)), "gpu_bpf_get_record")
        return r

    def get_ess(self) -> float:
        return self.get_record().ess

    def get_loglik_total(self) -> float:
        return self._lib.gpu_bpf_get_loglik_total(self._s)

    def set_loglik_semantics(self, mode: int) -> None:
        check(self._lib.gpu_bpf_set_loglik_semantics(self._s, int(mode)), "gpu_bpf_set_loglik_semantics")

    def get_particles(self):
        out = (C.c_float * self.n_particles)()
        check(self._lib.gpu_bpf_get_particles(self._s, out), "gpu_bpf_get_particles")
        return out

    def record_ancestors(self, enable: bool = True) -> None:
        check(self._lib.gpu_bpf_record_ancestors(self._s, int(enable)), "gpu_bpf_record_ancestors")

    def get_ancestors(self):
        """(resampled: bool, ancestors ctypes array of N int32)."""
        out = (C.c_int32 * self.n_particles)()
        rc = self._lib.gpu_bpf_get_ancestors(self._s, out)
        if rc < 0:
            raise BpfError(-rc, "gpu_bpf_get_ancestors")
        return bool(rc), out

    def get_resample_inputs(self):
        """(w[N] float32, tile_exp[ceil(N/4096)] int32, u23) of the last tick."""
        n = self.n_particles
        g = (n + 4095) // 4096
        w = (C.c_float * n)()
        te = (C.c_int32 * g)()
        u = C.c_uint32(0)
        check(self._lib.gpu_bpf_get_resample_inputs(self._s, w, te, C.byref(u)), "gpu_bpf_get_resample_inputs")
        return w, te, u.value

    def save(self) -> bytes:
        """Checkpoint of the filter's whole state (gpu_bpf_save)."""
        n = self._lib.gpu_bpf_checkpoint_bytes(self._s)
        buf = (C.c_ubyte * n)()
        check(self._lib.gpu_bpf_save(self._s, buf, n), "gpu_bpf_save")
        return bytes(buf)

    def load(self, blob: bytes) -> None:
        """Restore a checkpoint made by save() of a filter with the same particle count."""
        buf = (C.c_ubyte * len(blob)).from_buffer_copy(blob)
        check(self._lib.gpu_bpf_load(self._s, buf, len(blob)), "gpu_bpf_load")

    def set_fused_small(self, enable: bool = True) -> None:
        """Fused one-launch ticks for filters of at most 65536 particles (default on)."""
        check(self._lib.gpu_bpf_set_fused_small(self._s, int(bool(enable))), "gpu_bpf_set_fused_small")

    def profile(self, enable: bool = True) -> None:
        check(self._lib.gpu_bpf_profile(self._s, int(enable)), "gpu_bpf_profile")

    def profile_read(self):
        """(pass1_ms, plan_ms, pass2_ms, ticks) summed since profile(True)."""
        p1, pl, p2 = C.c_double(), C.c_double(), C.c_double()
        n1, n2 = C.c_int(), C.c_int()
        check(self._lib.gpu_bpf_profile_read(self._s, C.byref(p1), C.byref(pl), C.byref(p2), C.byref(n1),
                                             C.byref(n2)), "gpu_bpf_profile_read")
        return p1.value, pl.value, p2.value, n1.value


def debug_pcg32(seed: int, n: int, t: int):
    lib = _lib.load()
    out = (C.c_uint32 * n)()
    check(lib.gpu_bpf_debug_pcg32(int(seed), int(n), int(t), out), "gpu_bpf_debug_pcg32")
    return list(out)


def debug_normals(seed: int, n: int, t: int):
    lib = _lib.load()
    out = (C.c_float * n)()
    check(lib.gpu_bpf_debug_normals(int(seed), int(n), int(t), out), "gpu_bpf_debug_normals")
    return list(out)


def run_rmse(returns: Sequence[float], true_h: Sequence[float], n_particles: int, rho: float,
             sigma_z: float, mu: float, nu_state: float = 0.0, nu_obs: float = 0.0, seed: int = 42) -> float:
    lib = _lib.load()
    n = len(returns)
    ra = (C.c_double * n)(*returns)
    ha = (C.c_double * n)(*true_h)
    v = lib.gpu_bpf_run_rmse(ra, ha, n, int(n_particles), rho, sigma_z, mu, nu_state, nu_obs, int(seed))
    if math.isnan(v):
        raise BpfError(lib.gpu_bpf_last_error(), "gpu_bpf_run_rmse")
    return v
