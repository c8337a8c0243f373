"""Python face of the batched filter (include/gpu_bpf.h, "Batched filters")."""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional

from . import _lib
from ._lib import BpfBatchFilter, BpfError, check

SIZE_CLASS_MAX_N = (1024, 2048, 4096, 8192, 16384)


class GpuBpfBatch:
    """Many SV filters (own theta, N <= 16384, seed) on one observation series."""

    def __init__(self, filters: Iterable[dict], ess_threshold: float = 0.0):
        self._lib = _lib.load()
        fl = list(filters)
        arr = (BpfBatchFilter * len(fl))()
        for i, f in enumerate(fl):
            arr[i] = BpfBatchFilter(float(f["mu"]), float(f["rho"]), float(f["sigma_z"]),
                                    float(f.get("nu_obs", 0.0)), int(f["n_particles"]), int(f["seed"]),
                                    float(f.get("nu_state", 0.0)))
        h = self._lib.gpu_bpf_batch_create(arr, len(fl), float(ess_threshold))
        if not h:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_batch_create")
        self._h = h
        self.filters = fl
        self.n_filters = len(fl)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gpu_bpf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self._lib.gpu_bpf_batch_stream(self._h)

    def set_filters(self, filters: Iterable[dict]) -> None:
        """New (mu, rho, sigma_z, nu_obs, nu_state, seed) for every filter; each n_particles must equal
        the filter's count at creation (gpu_bpf_batch_set_filters)."""
        fl = list(filters)
        if len(fl) != self.n_filters:
            raise ValueError(f"expected {self.n_filters} filters, got {len(fl)}")
        arr = (BpfBatchFilter * len(fl))()
        for i, f in enumerate(fl):
            arr[i] = BpfBatchFilter(float(f["mu"]), float(f["rho"]), float(f["sigma_z"]),
                                    float(f.get("nu_obs", 0.0)), int(f["n_particles"]), int(f["seed"]),
                                    float(f.get("nu_state", 0.0)))
        check(self._lib.gpu_bpf_batch_set_filters(self._h, arr), "gpu_bpf_batch_set_filters")
        self.filters = fl

    def set_threads(self, size_class: int, threads: int) -> None:
        check(self._lib.gpu_bpf_batch_set_threads(self._h, int(size_class), int(threads)), "gpu_bpf_batch_set_threads")

    def get_threads(self, size_class: int) -> int:
        return self._lib.gpu_bpf_batch_get_threads(self._h, int(size_class))

    def autotune(self, y, n_ticks: Optional[int] = None, cache_path: Optional[str] = None) -> None:
        n = len(y) if n_ticks is None else int(n_ticks)
        ya = (C.c_float * n)(*[float(v) for v in y[:n]])
        check(self._lib.gpu_bpf_batch_autotune(self._h, ya, n, cache_path.encode() if cache_path else None),
              "gpu_bpf_batch_autotune")

    def run(self, y):
        """Host run: returns (loglik[B] list of float, hmean_last[B] list of float)."""
        n = len(y)
        ya = (C.c_float * n)(*[float(v) for v in y])
        ll = (C.c_double * self.n_filters)()
        hm = (C.c_float * self.n_filters)()
        check(self._lib.gpu_bpf_batch_run(self._h, ya, n, ll, hm), "gpu_bpf_batch_run")
        return list(ll), list(hm)

    def run_device(self, y_ptr: int, n_ticks: int, loglik_ptr: int, dll_ptr: int = 0, hmean_ptr: int = 0) -> None:
        check(self._lib.gpu_bpf_batch_run_device(self._h, C.c_void_p(y_ptr), int(n_ticks), C.c_void_p(loglik_ptr),
                                                 C.c_void_p(dll_ptr or None), C.c_void_p(hmean_ptr or None)),
              "gpu_bpf_batch_run_device")

    def run_debug(self, y_ptr: int, n_ticks: int, loglik_ptr: int, dll_ptr: int = 0, anc_ptr: int = 0,
                  particles_ptr: int = 0) -> None:
        check(self._lib.gpu_bpf_batch_run_debug(self._h, C.c_void_p(y_ptr), int(n_ticks), C.c_void_p(loglik_ptr),
                                                C.c_void_p(dll_ptr or None), C.c_void_p(anc_ptr or None),
                                                C.c_void_p(particles_ptr or None)), "gpu_bpf_batch_run_debug")

    def run_correlated(self, y_ptr: int, n_ticks: int, noise_in_ptr: int, noise_out_ptr: int, rho: float,
                       loglik_ptr: int, dll_ptr: int = 0, anc_ptr: int = 0) -> None:
        """Correlated-noise run from tick 0 (device pointers, batch stream): noise_out receives the
        noise used, rho * noise_in + sqrt(1 - rho^2) * fresh (noise_in 0: fresh only). Areas start
        at noise_offset(f, n_ticks) floats; see gpu_bpf_batch_run_correlated."""
        check(self._lib.gpu_bpf_batch_run_correlated(self._h, C.c_void_p(y_ptr), int(n_ticks),
                                                     C.c_void_p(noise_in_ptr or None), C.c_void_p(noise_out_ptr),
                                                     float(rho), C.c_void_p(loglik_ptr), C.c_void_p(dll_ptr or None),
                                                     C.c_void_p(anc_ptr or None)), "gpu_bpf_batch_run_correlated")

    def noise_offset(self, f: int, n_ticks: int) -> int:
        """First float of filter f's noise area (f = n_filters: the buffers' length)."""
        v = int(self._lib.gpu_bpf_batch_noise_offset(self._h, int(f), int(n_ticks)))
        if v < 0:
            raise BpfError(-v, "gpu_bpf_batch_noise_offset")
        return v

    def grad_run(self, y_ptr: int, n_ticks: int, loglik_ptr: int, grad_ptr: int) -> None:
        """Forward + adjoint backward of every filter: loglik[B] (FP64) and grad[B, 3] = d loglik /
        d(mu, rho, sigma_z), enqueued on the batch stream (device pointers)."""
        check(self._lib.gpu_bpf_batch_grad_run(self._h, C.c_void_p(y_ptr), int(n_ticks), C.c_void_p(loglik_ptr),
                                               C.c_void_p(grad_ptr)), "gpu_bpf_batch_grad_run")

    def step_device(self, y_ptr: int, n_ticks: int, dll_ptr: int = 0, hmean_ptr: int = 0) -> None:
        """Advance every filter n_ticks from its saved state (device pointers, batch stream)."""
        check(self._lib.gpu_bpf_batch_step_device(self._h, C.c_void_p(y_ptr), int(n_ticks), C.c_void_p(dll_ptr or None),
                                                  C.c_void_p(hmean_ptr or None)), "gpu_bpf_batch_step_device")

    def reset(self) -> None:
        check(self._lib.gpu_bpf_batch_reset(self._h), "gpu_bpf_batch_reset")

    @property
    def tick(self) -> int:
        return self._lib.gpu_bpf_batch_tick(self._h)

    @property
    def loglik_ptr(self) -> int:
        return self._lib.gpu_bpf_batch_loglik_device(self._h)

    def grad_tape_bytes(self, n_ticks: int) -> int:
        return int(self._lib.gpu_bpf_batch_grad_tape_bytes(self._h, int(n_ticks)))

    def resample_counts(self):
        cnt = (C.c_int * self.n_filters)()
        hm = (C.c_float * self.n_filters)()
        check(self._lib.gpu_bpf_batch_resample_counts(self._h, cnt, hm), "gpu_bpf_batch_resample_counts")
        return list(cnt), list(hm)
