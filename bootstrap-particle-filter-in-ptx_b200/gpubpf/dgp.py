"""Synthetic stochastic-volatility series (the reference's matched DGP).

Restates ``generate_matched_series`` and its PCG32 helpers from the reference
test ``tests/test_bpf_matched_dgp.cu`` (seeding :69-76, doubles :78-80,
Box-Muller :82-87, Student-t :89-99, series :141-175), plus the series used by
the benchmark configurations.
"""
from __future__ import annotations

import math

MASK64 = (1 << 64) - 1
PCG_MULT = 6364136223846793005


class Pcg32:
    """PCG32 with explicit increment (test_bpf_matched_dgp.cu:59-76)."""

    def __init__(self, seed: int):
        self.state = 0
        self.inc = ((seed * 12345) | 1) & MASK64
        self.next_u32()
        self.state = (self.state + seed * 67890) & MASK64
        self.next_u32()
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * PCG_MULT + self.inc) & MASK64
        xsh = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xsh >> rot) | (xsh << ((-rot) & 31))) & 0xFFFFFFFF

    def next_double(self) -> float:          # :78-80, 21-bit uniform in [0,1)
        return (self.next_u32() >> 11) * (1.0 / 2097152.0)

    def gaussian(self) -> float:             # :82-87
        while True:
            u1 = self.next_double()
            if u1 >= 1e-10:
                break
        u2 = self.next_double()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * 3.14159265358979323846 * u2)

    def student_t(self, nu: float) -> float:  # :89-99: z / sqrt(chi2 / nu), chi2 with int(nu) dof
        if nu > 100.0:
            return self.gaussian()
        z = self.gaussian()
        chi_sq = 0.0
        for _ in range(int(nu)):
            g = self.gaussian()
            chi_sq += g * g
        return z / math.sqrt(chi_sq / nu)


def matched_series(T: int, rho: float, sigma_z: float, mu: float, seed: int, nu_state: float = 0.0,
                   nu_obs: float = 0.0):
    """(true_h[T], y[T]) from generate_matched_series; nu_state / nu_obs > 0 draw the state /
    observation noise from Student-t laws (0 = Gaussian)."""
    rng = Pcg32(seed)
    var_stat = (sigma_z * sigma_z) / max(1.0 - rho * rho, 1e-6)
    h = mu + math.sqrt(var_stat) * rng.gaussian()
    hs, ys = [], []
    for t in range(T):
        if t > 0:
            eps = rng.student_t(nu_state) if nu_state > 0.0 else rng.gaussian()
            h = mu + rho * (h - mu) + sigma_z * eps
        h = min(max(h, -12.0), 4.0)
        hs.append(h)
        eta = rng.student_t(nu_obs) if nu_obs > 0.0 else rng.gaussian()
        ys.append(math.exp(h / 2.0) * eta)
    return hs, ys


def regime_series(T: int, mus=(-1.5, 0.0), period: int = 500, rho: float = 0.97,
                  sigma_z: float = 0.2, seed: int = 42):
    """Regime-switching SV series: mu alternates every `period` ticks, same DGP otherwise."""
    rng = Pcg32(seed)
    mu0 = mus[0]
    var_stat = (sigma_z * sigma_z) / max(1.0 - rho * rho, 1e-6)
    h = mu0 + math.sqrt(var_stat) * rng.gaussian()
    hs, ys = [], []
    for t in range(T):
        mu = mus[(t // period) % len(mus)]
        if t > 0:
            h = mu + rho * (h - mu) + sigma_z * rng.gaussian()
        h = min(max(h, -12.0), 4.0)
        hs.append(h)
        ys.append(math.exp(h / 2.0) * rng.gaussian())
    return hs, ys


def cond_resample_series(sigma_of_t, T: int = 3000, rho: float = 0.98, mu: float = -4.5, seed: int = 42):
    """(true_h[T], y[T]) of the reference's conditional-resampling study (tests/test_cond_resample.cu:
    25-57): its host PCG32 (fixed increment) and FP32 Box-Muller, h_0 = mu, sigma_z = sigma_of_t(t)
    (the regime scenario changes it mid-series). Restated in numpy FP32; the same law as the C
    build, not pinned to it bit for bit."""
    import numpy as np
    f32 = np.float32
    state = seed

    def u23():
        nonlocal state
        old = state
        state = (old * PCG_MULT + 1442695040888963407) & MASK64
        xsh = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        r = ((xsh >> rot) | (xsh << ((-rot) & 31))) & 0xFFFFFFFF
        return f32(r >> 9) * f32(1.0 / 8388608.0)

    def randn():
        u1 = u23() + f32(1e-10)
        u2 = u23()
        return f32(np.sqrt(f32(-2.0) * np.log(f32(u1)))) * f32(np.cos(f32(2.0) * f32(3.14159265358979) * u2))

    h = f32(mu)
    ys, hs = [], []
    for t in range(T):
        h = f32(mu) + f32(rho) * (h - f32(mu)) + f32(sigma_of_t(t)) * randn()
        ys.append(float(f32(np.exp(h * f32(0.5))) * randn()))
        hs.append(float(h))
    return np.array(hs), np.array(ys, dtype=np.float32)
