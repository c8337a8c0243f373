"""Parameter tables of the benchmark configurations.

Batched configurations draw each filter's theta and particle count from a
host PCG32 (the matched-DGP generator of the reference test
tests/test_bpf_matched_dgp.cu:59-87) seeded with 4:
  mu ~ N(-1, 0.5^2), phi ~ U(0.85, 0.995), sigma_eta ~ U(0.05, 0.4),
  N = round(exp(U(ln 512, ln 16384))) (configuration 4; configuration 5 uses N = 8192).
Filter b gets the PCG32 seed 1000 + b.
"""
from __future__ import annotations

import math

from .dgp import Pcg32


def batch_thetas(B: int, n_fixed: int | None = None, seed: int = 4):
    """List of dicts (mu, rho, sigma_z, n_particles, seed) for B filters."""
    rng = Pcg32(seed)
    out = []
    lo, hi = math.log(512.0), math.log(16384.0)
    for b in range(B):
        mu = -1.0 + 0.5 * rng.gaussian()
        rho = 0.85 + (0.995 - 0.85) * rng.next_double()
        sig = 0.05 + (0.4 - 0.05) * rng.next_double()
        u = rng.next_double()
        n = n_fixed if n_fixed is not None else int(round(math.exp(lo + (hi - lo) * u)))
        out.append({"mu": mu, "rho": rho, "sigma_z": sig, "n_particles": max(1, min(16384, n)),
                    "seed": 1000 + b, "nu_obs": 0.0})
    return out


def config4(B: int = 1024):
    """Batched SMC2-style inner loop: 1024 filters, N log-uniform in [512, 16384]."""
    return batch_thetas(B)


def config5(B: int = 256):
    """Batched + gradient: 256 filters with N = 8192."""
    return batch_thetas(B, n_fixed=8192)
