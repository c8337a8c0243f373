"""Python face of the SMC^2 driver (include/gpu_bpf.h, "SMC^2 over the SV parameters";
the outer loop of the reference's smc2_cuda_* API, smc2/smc2_rbpf_batch.cuh:461-489)."""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _lib
from ._lib import BpfError, BpfSmc2Prior, check


class Smc2:
    """Online posterior over theta = (mu, rho, sigma_z) of the SV model."""

    def __init__(self, n_theta: int, n_particles: int, max_ticks: int, prior: Optional[dict] = None,
                 seed: int = 1):
        self._lib = _lib.load()
        pp = None
        if prior is not None:
            pp = BpfSmc2Prior(prior["mu_mean"], prior["mu_sd"], prior["rho_lo"], prior["rho_hi"],
                              prior["sigma_lo"], prior["sigma_hi"])
        h = self._lib.gpu_bpf_smc2_create(int(n_theta), int(n_particles), int(max_ticks),
                                          C.byref(pp) if pp is not None else None, int(seed))
        if not h:
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_smc2_create")
        self._h = h
        self.n_theta = int(n_theta)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gpu_bpf_smc2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_moves(self, n_moves: int = 1, outer_ess_threshold: float = 0.5, proposal_scale: float = 1.0) -> None:
        check(self._lib.gpu_bpf_smc2_set_moves(self._h, int(n_moves), float(outer_ess_threshold),
                                               float(proposal_scale)), "gpu_bpf_smc2_set_moves")

    def update(self, y: float) -> float:
        ess = self._lib.gpu_bpf_smc2_update(self._h, float(y))
        if math.isnan(ess):
            raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_smc2_update")
        return ess

    def theta(self):
        m, s = (C.c_float * 3)(), (C.c_float * 3)()
        check(self._lib.gpu_bpf_smc2_get_theta(self._h, m, s), "gpu_bpf_smc2_get_theta")
        return np.array(list(m)), np.array(list(s))

    def particles(self):
        th = np.zeros((self.n_theta, 3), dtype=np.float32)
        lw = np.zeros(self.n_theta)
        ll = np.zeros(self.n_theta)
        check(self._lib.gpu_bpf_smc2_get_particles(self._h, th.ctypes.data, lw.ctypes.data, ll.ctypes.data),
              "gpu_bpf_smc2_get_particles")
        return th, lw, ll

    def set_cpmmh_rho(self, rho: float) -> None:
        """Correlated-noise PMMH moves with correlation rho (0 = fresh inner filters, the default;
        ~ smc2_cuda_set_cpmmh_rho). Switch on or off before the first update."""
        check(self._lib.gpu_bpf_smc2_set_cpmmh_rho(self._h, float(rho)), "gpu_bpf_smc2_set_cpmmh_rho")

    def last_move(self):
        """The last PMMH move: dict of theta_prop, theta_cur [M, 3] (float32, as the inner filters
        use them), loglik_prop, loglik_cur [M] and accepted [M]."""
        M = self.n_theta
        tp = np.zeros((M, 3), dtype=np.float32)
        tc = np.zeros((M, 3), dtype=np.float32)
        lp = np.zeros(M)
        lc = np.zeros(M)
        acc = np.zeros(M, dtype=np.int32)
        check(self._lib.gpu_bpf_smc2_get_last_move(self._h, tp.ctypes.data, tc.ctypes.data, lp.ctypes.data,
                                                   lc.ctypes.data, acc.ctypes.data), "gpu_bpf_smc2_get_last_move")
        return {"theta_prop": tp, "theta_cur": tc, "loglik_prop": lp, "loglik_cur": lc, "accepted": acc}

    def last_update(self):
        """The last update: dict of dll [M] (the forward tick's inner log-likelihood increments),
        resampled (bool) and ancestors [M] (the outer ancestors when resampled, else None)."""
        M = self.n_theta
        dll = np.zeros(M)
        res = C.c_int(0)
        anc = np.zeros(M, dtype=np.int32)
        check(self._lib.gpu_bpf_smc2_get_last_update(self._h, dll.ctypes.data, C.addressof(res), anc.ctypes.data),
              "gpu_bpf_smc2_get_last_update")
        return {"dll": dll, "resampled": bool(res.value), "ancestors": anc if res.value else None}

    def noise(self, j: int, n_ticks: int, n_particles: int):
        """Theta-particle j's current auxiliary noise: (normals [n_ticks, n_particles], resampling
        normals [n_ticks])."""
        stride = ((n_particles + 3) & ~3) + 4
        out = np.zeros((n_ticks, stride), dtype=np.float32)
        check(self._lib.gpu_bpf_smc2_get_noise(self._h, int(j), int(n_ticks), out.ctypes.data),
              "gpu_bpf_smc2_get_noise")
        return out[:, :n_particles].copy(), out[:, stride - 4].copy()

    def stats(self):
        r, p, a = C.c_int(0), C.c_longlong(0), C.c_longlong(0)
        check(self._lib.gpu_bpf_smc2_stats(self._h, C.byref(r), C.byref(p), C.byref(a)), "gpu_bpf_smc2_stats")
        return {"rejuvenations": r.value, "proposed": p.value, "accepted": a.value}
