"""Host restatement of the SMC^2 outer loop (TEST INFRASTRUCTURE ONLY: the checker of
gpu_bpf_smc2_*; the product never imports it).

Restates, in plain Python on doubles, the outer step of the reference's smc2_cuda_update
(smc2/smc2_rbpf_batch.cu:1329-1502) as this build's driver applies it to the SV parameters
theta = (mu, rho, sigma_z):

  outer weights   logw_j += the inner filter's log-likelihood increment of the tick
                  (the inner step before smc2_rbpf_batch.cu:1365)
  outer ESS       (sum w)^2 / sum w^2 over w_j = exp(logw_j - max logw) (:1365-1372)
  resampling      systematic, one uniform, ancestors a_j = min{k : C_k > (u + j) / M C_M}
                  (:1372-1401); copies keep their parent's theta, log-weights reset to 0
                  (:1477)
  PMMH move       random walk with covariance 2.38^2 / 3 * scale * (empirical covariance of
                  the theta-particles) via its Cholesky factor, prior log-density of current
                  and proposed theta, acceptance log u < ll' + lp' - ll - lp (:1446-1475)

The inner log-likelihoods come from the device (the inner filters are the product's
batched kernel; their parity is tested elsewhere), so the checks here are of the outer
loop's own arithmetic: every draw of the driver's host PCG32 stream, the ESS, the
ancestors, the proposals and the acceptance flags.
"""
from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1
PCG_A = 6364136223846793005
PRIOR_DEFAULT = (-1.0, 0.5, 0.85, 0.995, 0.05, 0.4)   # mu_mean, mu_sd, rho_lo, rho_hi, sigma_lo, sigma_hi


class HostPcg:
    """PCG32 (O'Neill 2014), XSH-RR output of the pre-step state; 53-bit uniforms from two draws,
    Box-Muller normals."""

    def __init__(self, seed: int, stream: int):
        self.inc = ((stream << 1) | 1) & M64
        self.s = 0
        self.next()
        self.s = (self.s + seed) & M64
        self.next()

    def next(self) -> int:
        old = self.s
        self.s = (old * PCG_A + self.inc) & M64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF

    def uniform(self) -> float:
        a = self.next() >> 5
        b = self.next() >> 6
        return (float(a) * 67108864.0 + float(b) + 0.5) / 9007199254740992.0

    def normal(self) -> float:
        u1 = self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586476925286766559 * u2)


def f32(x: float) -> float:
    return float(np.float32(x))


class Smc2Outer:
    """The driver's outer loop on given inner log-likelihoods."""

    def __init__(self, n_theta: int, seed: int, prior=None, n_moves: int = 1, ess_frac: float = 0.5,
                 scale: float = 1.0):
        self.M = int(n_theta)
        # the prior's fields are floats in the C struct
        self.prior = tuple(f32(v) for v in (prior or PRIOR_DEFAULT))
        self.n_moves = n_moves
        self.ess_frac = f32(ess_frac)
        self.scale = f32(scale)
        self.rng = HostPcg(seed, 0x5EED)
        self.next_seed = (seed & 0x3FFFFFFF) + 1
        mu_mean, mu_sd, rho_lo, rho_hi, s_lo, s_hi = self.prior
        self.theta = []
        for _ in range(self.M):
            mu = mu_mean + mu_sd * self.rng.normal()
            # (hi - lo) is a single-precision difference in the driver (float fields)
            rho = rho_lo + f32(rho_hi - rho_lo) * self.rng.uniform()
            sig = s_lo + f32(s_hi - s_lo) * self.rng.uniform()
            self.theta.append((mu, rho, sig))
            self.next_seed += 1
        self.logw = [0.0] * self.M

    def log_prior(self, th) -> float:
        mu_mean, mu_sd, rho_lo, rho_hi, s_lo, s_hi = self.prior
        mu, rho, sig = th
        if not (rho > rho_lo and rho < rho_hi and sig > s_lo and sig < s_hi):
            return -math.inf
        z = (mu - mu_mean) / mu_sd
        return (-0.5 * z * z - math.log(mu_sd) - math.log(f32(rho_hi - rho_lo)) - math.log(f32(s_hi - s_lo))
                - 0.918938533204672741780329736406)

    def outer_ess(self) -> float:
        m = -math.inf
        for v in self.logw:
            m = max(m, v)
        a = b = 0.0
        for v in self.logw:
            e = math.exp(v - m)
            a += e
            b += e * e
        return a * a / b

    def observe(self, dll):
        """Adds one tick's inner increments; returns (ESS, whether the loop resamples now)."""
        for j in range(self.M):
            self.logw[j] += float(dll[j])
        ess = self.outer_ess()
        return ess, ess < float(self.ess_frac) * self.M

    def resample(self):
        """Systematic resampling of the theta-particles; returns the ancestors."""
        M = self.M
        m = -math.inf
        for v in self.logw:
            m = max(m, v)
        cdf, acc = [], 0.0
        for v in self.logw:
            acc += math.exp(v - m)
            cdf.append(acc)
        u0 = self.rng.uniform()
        idx, k = [], 0
        for j in range(M):
            tgt = (u0 + j) / M * acc
            while k < M - 1 and cdf[k] <= tgt:
                k += 1
            idx.append(k)
        self.next_seed += M
        self.theta = [self.theta[i] for i in idx]
        self.logw = [0.0] * M
        return idx

    def propose(self):
        """One PMMH proposal per theta-particle. Returns (theta scored by each proposal's inner
        filter, as float32 [M, 3]; the current theta as float32 [M, 3])."""
        M = self.M
        c = float(self.scale) * 2.38 * 2.38 / 3.0
        mean = [0.0, 0.0, 0.0]
        for q in self.theta:
            for a in range(3):
                mean[a] += q[a]
        mean = [v / M for v in mean]
        cov = [[0.0] * 3 for _ in range(3)]
        for q in self.theta:
            d = [q[0] - mean[0], q[1] - mean[1], q[2] - mean[2]]
            for a in range(3):
                for b in range(3):
                    cov[a][b] += d[a] * d[b] / M
        L = [[0.0] * 3 for _ in range(3)]
        for a in range(3):
            for b in range(a + 1):
                v = c * cov[a][b] + (1e-10 if a == b else 0.0)
                for q in range(b):
                    v -= L[a][q] * L[b][q]
                L[a][b] = math.sqrt(max(v, 1e-12)) if a == b else v / L[b][b]
        self._pr, self._lp, self._lpn = [], [], []
        scored = np.zeros((M, 3), dtype=np.float32)
        cur = np.zeros((M, 3), dtype=np.float32)
        for j in range(M):
            z = [self.rng.normal(), self.rng.normal(), self.rng.normal()]
            d0 = L[0][0] * z[0]
            d1 = L[1][0] * z[0] + L[1][1] * z[1]
            d2 = L[2][0] * z[0] + L[2][1] * z[1] + L[2][2] * z[2]
            th = self.theta[j]
            pr = (th[0] + d0, th[1] + d1, th[2] + d2)
            lp, lpn = self.log_prior(th), self.log_prior(pr)
            self._pr.append(pr)
            self._lp.append(lp)
            self._lpn.append(lpn)
            self.next_seed += 1
            scored[j] = pr if math.isfinite(lpn) else th
            cur[j] = th
        return scored, cur

    def accept(self, ll_prop, ll_cur):
        """Acceptance flags of the last proposals given the proposals' and current inner total
        log-likelihoods; accepted thetas become current."""
        flags = []
        for j in range(self.M):
            la = float(ll_prop[j]) + self._lpn[j] - float(ll_cur[j]) - self._lp[j]
            ok = math.isfinite(self._lpn[j]) and math.isfinite(float(ll_prop[j])) and math.log(self.rng.uniform()) < la
            flags.append(1 if ok else 0)
            if ok:
                self.theta[j] = self._pr[j]
        return flags

    def theta_f32(self):
        return np.asarray(self.theta, dtype=np.float32)
