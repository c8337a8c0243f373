"""Python face of the IMM entry points (include/gpu_bpf.h, "IMM"; the reference's
gpu_imm_* API, gpu_bpf/gpu_bpf.cuh:131-164)."""
from __future__ import annotations

import ctypes as C
import math
from typing import Iterable, Optional, Sequence

from . import _lib
from ._lib import BpfError, ImmModelParams


class Imm:
    """K SV models with Markov model switching, stepped one observation at a time."""

    def __init__(self, models: Iterable[dict], n_particles_per_model: int,
                 transition_matrix: Optional[Sequence[float]] = None, seed: int = 42):
        self._lib = _lib.load()
        ml = list(models)
        arr = (ImmModelParams * len(ml))()
        for i, m in enumerate(ml):
            arr[i] = ImmModelParams(float(m["rho"]), float(m["sigma_z"]), float(m["mu"]),
                                    float(m.get("nu_state", 0.0)), float(m.get("nu_obs", 0.0)))
        tm = None
        if transition_matrix is not None:
            tm = (C.c_float * len(transition_matrix))(*[float(v) for v in transition_matrix])
        h = self._lib.gpu_imm_create(arr, len(ml), int(n_particles_per_model), tm, int(seed))
        if not h:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_imm_create")
        self._h = h
        self.n_models = len(ml)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gpu_imm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, y_t: float):
        r = self._lib.gpu_imm_step(self._h, float(y_t))
        if math.isnan(r.h_mean):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_imm_step")
        return r

    def probs(self):
        out = (C.c_float * self.n_models)()
        self._lib.gpu_imm_get_probs(self._h, out)
        return list(out)

    @property
    def state(self):
        return self._h.contents


def build_grid(rhos, sigma_zs, mus, nu_state: float = 0.0, nu_obs: float = 0.0):
    """gpu_imm_build_grid: list of model dicts in the reference's rho-major order."""
    lib = _lib.load()
    fa = lambda v: (C.c_float * len(v))(*[float(x) for x in v])
    n = C.c_int(0)
    p = lib.gpu_imm_build_grid(fa(rhos), len(rhos), fa(sigma_zs), len(sigma_zs), fa(mus), len(mus),
                               float(nu_state), float(nu_obs), C.byref(n))
    if not p:
        raise BpfError(lib.gpu_bpf_last_error(), "gpu_imm_build_grid")
    out = [{"rho": p[i].rho, "sigma_z": p[i].sigma_z, "mu": p[i].mu, "nu_state": p[i].nu_state,
            "nu_obs": p[i].nu_obs} for i in range(n.value)]
    C.CDLL(None).free(C.cast(p, C.c_void_p))
    return out
