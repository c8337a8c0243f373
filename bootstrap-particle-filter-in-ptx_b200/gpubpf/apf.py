"""Auxiliary particle filter (gpu_apf_* of include/gpu_bpf.h; reference gpu_bpf/gpu_bpf.cuh:114-126)."""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

from . import _lib
from ._lib import BpfError, BpfResult, BpfTickRecord, check


class GpuApf:
    """Two-stage auxiliary particle filter on the plain filter's kernels.

    ``step`` returns the reference's ``BpfResult`` (``log_lik`` = log mean of the second-stage
    weights); ``get_record().dloglik`` is the APF estimate of log p(y_t | y_1:t-1)."""

    def __init__(self, n_particles: int, rho: float, sigma_z: float, mu: float,
                 nu_state: float = 0.0, nu_obs: float = 0.0, seed: int = 42):
        self._lib = _lib.load()
        self._s = self._lib.gpu_apf_create(int(n_particles), rho, sigma_z, mu, nu_state, nu_obs, int(seed))
        if not self._s:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_apf_create")
        self.n_particles = int(n_particles)

    def close(self) -> None:
        if getattr(self, "_s", None):
            self._lib.gpu_apf_destroy(self._s)
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
    def state(self) -> _lib.GpuApfState:
        return self._s.contents

    def step(self, y_t: float) -> BpfResult:
        r = self._lib.gpu_apf_step(self._s, float(y_t))
        if math.isnan(r.h_mean):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_apf_step")
        return r

    def step_many(self, y: Sequence[float], records: bool = False):
        n = len(y)
        ya = (C.c_float * n)(*y)
        if records:
            rec = (BpfTickRecord * n)()
            check(self._lib.gpu_apf_step_many(self._s, ya, n, None, rec), "gpu_apf_step_many")
            return list(rec)
        out = (BpfResult * n)()
        check(self._lib.gpu_apf_step_many(self._s, ya, n, out, None), "gpu_apf_step_many")
        return list(out)

    def get_record(self) -> BpfTickRecord:
        r = BpfTickRecord()
        check(self._lib.gpu_apf_get_record(self._s, C.byref(r)), "gpu_apf_get_record")
        return r

    def get_loglik_total(self) -> float:
        v = self._lib.gpu_apf_get_loglik_total(self._s)
        if math.isnan(v):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_apf_get_loglik_total")
        return v

    def get_particles(self):
        out = (C.c_float * self.n_particles)()
        check(self._lib.gpu_apf_get_particles(self._s, out), "gpu_apf_get_particles")
        return out

    def record_ancestors(self, enable: bool = True) -> None:
        check(self._lib.gpu_apf_record_ancestors(self._s, int(bool(enable))), "gpu_apf_record_ancestors")

    def get_ancestors(self):
        """(first-stage ancestors, second-stage ancestors) of the last tick."""
        a1 = (C.c_int32 * self.n_particles)()
        a2 = (C.c_int32 * self.n_particles)()
        check(self._lib.gpu_apf_get_ancestors(self._s, a1, a2), "gpu_apf_get_ancestors")
        return a1, a2


def apf_run_rmse(returns: Sequence[float], true_h: Sequence[float], n_particles: int, rho: float,
                 sigma_z: float, mu: float, nu_state: float = 0.0, nu_obs: float = 0.0, seed: int = 42) -> float:
    lib = _lib.load()
    n = len(returns)
    ra = (C.c_double * n)(*returns)
    ha = (C.c_double * n)(*true_h)
    v = lib.gpu_apf_run_rmse(ra, ha, n, int(n_particles), rho, sigma_z, mu, nu_state, nu_obs, int(seed))
    if math.isnan(v):
        raise BpfError(lib.gpu_bpf_last_error(), "gpu_apf_run_rmse")
    return v
