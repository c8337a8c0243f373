"""GPU tests of online mu / rho learning (gpu_bpf_enable_mu_learning and friends).

  score sums vs a host restatement      <= 1e-4 relative (FP32 particles and weights, FP64 sums)
  (PTX :1187-1227: sum W dlw, sum W dlw^2,
  sum W dlw dh, sum W dlw^2 dh^2)
  update rule vs a host restatement     <= 1e-5 relative on mu and rho (the reference's formulas,
  (gpu_bpf_ptx_full.cu:489-543)         fed the same sums)
  learning from a wrong mu              moves mu most of the way to the generating value
  the reference's mu-regime head-to-head  learning lowers the phase-2 RMSE; learnt mu and phase-2
  (smc2/test_mu_learning.cu:232-290)      RMSE within 0.1 / 0.02 of the reference's own learning
                                          filter on the same series
  the reference's rho-regime test         mu + rho learning: learnt rho within 0.02, mu within 0.1,
  (smc2/test_mu_learning.cu:468-525)      phase-2 RMSE within 0.02 of the reference's
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def _series(T, seed=42, mu=MU):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, RHO, SIG, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def _host_sums(f, h_prev, y, mu, nu_obs):
    w, te, _ = f.get_resample_inputs()
    w = np.frombuffer(w, dtype=np.float32).astype(np.float64)
    te = np.frombuffer(te, dtype=np.int32)
    N = w.shape[0]
    scale = np.repeat(np.exp2(te.astype(np.float64) - te.max()), 4096)[:N]
    W = w * scale
    W /= W.sum()
    h = np.frombuffer(f.get_particles(), dtype=np.float32).astype(np.float64)
    q = float(y) ** 2 * np.exp(-h)
    dlw = -0.5 + 0.5 * q if nu_obs == 0.0 else -0.5 + 0.5 * (nu_obs + 1.0) * (q / nu_obs) / (1.0 + q / nu_obs)
    dh = h_prev - mu
    return np.array([np.sum(W * dlw), np.sum(W * dlw ** 2), np.sum(W * dlw * dh), np.sum(W * dlw ** 2 * dh ** 2)]), h


@pytest.mark.parametrize("nu_obs", [0.0, 5.0])
def test_score_sums_match_host(bpf, nu_obs):
    N = 20000
    y = _series(4)
    f = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, nu_obs, 3, ess_threshold=1e-12)   # no resampling
    f.enable_mu_learning(1, 1000, 0.1, 10.0, 0.667)
    f.step(float(y[0]))
    h_prev = np.frombuffer(f.get_particles(), dtype=np.float32).astype(np.float64)
    sums, n = f.learning_sums()
    assert n == 0 and sums == [0.0, 0.0, 0.0, 0.0]                    # tick 0 has no transition
    expect = np.zeros(4)
    for t in (1, 2):
        f.step(float(y[t]))
        assert f.get_record().resampled == 0
        v, h_prev = _host_sums(f, h_prev, y[t], MU, nu_obs)
        expect += v
        sums, n = f.learning_sums()
        assert n == t
        np.testing.assert_allclose(sums, expect, rtol=1e-4, atol=1e-9)
    f.close()


def test_update_rule_matches_reference_formulas(bpf):
    N, K, c, t0, gamma = 8192, 4, 0.3, 10.0, 0.667
    y = _series(8)
    mu0, rho0 = -0.6, 0.95
    a = bpf.GpuBpf(N, rho0, SIG, mu0, 0.0, 0.0, 5, ess_threshold=0.5)
    b = bpf.GpuBpf(N, rho0, SIG, mu0, 0.0, 0.0, 5, ess_threshold=0.5)
    a.enable_mu_learning(1, 1000, c, t0, gamma)
    b.enable_mu_learning(1, K, c, t0, gamma)
    a.enable_rho_learning(True)
    b.enable_rho_learning(True)
    for t in range(K + 1):                  # ticks 1..K accumulate; b updates after tick K
        a.step(float(y[t]))
        b.step(float(y[t]))
    sums, n = a.learning_sums()
    assert n == K
    eta = c / (1 + t0) ** gamma

    def step(g, fi):
        mg, mf = g / K, fi / K
        d = mg / max(mf, 1e-8)
        if abs(d) > 5.0:
            d *= 5.0 / abs(d)
        snr = abs(mg) / max(math.sqrt(mf / K), 1e-10)
        return eta * min(snr / 2.0, 1.0) * d
    rho_f = float(np.float32(rho0))
    alpha = float(np.float32(mu0)) * (1 - rho_f) + step(sums[0], sums[1])
    mu_exp = min(max(alpha / max(1 - rho_f, 1e-6), -5.0), 2.0)
    rho_exp = min(max(rho_f + step(sums[2], sums[3]), 0.001), 0.999)
    assert abs(b.get_mu() - mu_exp) <= 1e-5 * max(1.0, abs(mu_exp)), (b.get_mu(), mu_exp)
    assert abs(b.get_rho() - rho_exp) <= 1e-5, (b.get_rho(), rho_exp)
    assert a.get_mu() == np.float32(mu0)
    s2, n2 = b.learning_sums()
    assert n2 == 0 and s2 == [0.0, 0.0, 0.0, 0.0]
    b.set_mu(-1.0)                          # an external push restarts the schedule
    assert b.learning_sums()[1] == 0
    a.close()
    b.close()


def test_mu_learning_moves_to_the_generating_value(bpf):
    y = _series(2000, seed=8, mu=-1.0)
    f = bpf.GpuBpf(8192, RHO, SIG, 0.0, 0.0, 0.0, 11, ess_threshold=0.5)   # starts at mu = 0
    f.enable_mu_learning(1, 25, 1.0, 10.0, 0.667)
    recs = f.step_many(y.tolist(), records=True)
    assert len(recs) == len(y)
    mu = f.get_mu()
    f.disable_mu_learning()
    f.close()
    assert abs(mu - (-1.0)) < 0.4, mu


def _mu_regime_series(T=5000, t_switch=2500, mu1=-1.0, mu2=-2.5, rho=0.98, sigma_z=0.15, nu_obs=5.0, seed=42,
                      rho2=None):
    """generate_sv_mu_regime of smc2/test_mu_learning.cu:70-108 (FP64, its host PCG32 + Box-Muller:
    all state draws first, then all observation draws); with rho2, generate_sv_rho_regime
    (:110-140): mu1 throughout, rho -> rho2 at t_switch."""
    rng = seed

    def randn():
        nonlocal rng
        s = (rng * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        u1 = (s >> 11) * (1.0 / 9007199254740992.0)
        s = (s * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        u2 = (s >> 11) * (1.0 / 9007199254740992.0)
        rng = s
        u1 = max(u1, 1e-15)
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * 3.14159265358979323846 * u2)

    def sample_t(nu):
        z = randn()
        chi2 = 0.0
        for _ in range(int(nu)):
            g = randn()
            chi2 += g * g
        return z / math.sqrt(chi2 / nu)

    h = np.zeros(T)
    h[0] = mu1 + sigma_z / math.sqrt(max(1.0 - rho * rho, 1e-10)) * randn()
    for t in range(1, T):
        if rho2 is None:
            mu, r = (mu1 if t < t_switch else mu2), rho
        else:
            mu, r = mu1, (rho if t < t_switch else rho2)
        h[t] = mu + r * (h[t - 1] - mu) + sigma_z * randn()
    y = np.array([math.exp(h[t] / 2.0) * sample_t(nu_obs) for t in range(T)], dtype=np.float32)
    return h, y


def test_mu_regime_head_to_head_with_reference(bpf):
    """The reference's head-to-head test (smc2/test_mu_learning.cu:232-290): mu shifts from -1.0
    to -2.5 at t = 2500 (rho 0.98, sigma_z 0.15, nu_obs 5, N = 4096, T = 5000); both filters start
    at mu = -1.0, one without learning, one with natural-gradient learning (K 50, c 0.1, t0 10,
    gamma 2/3). Learning lowers the phase-2 RMSE; the learnt mu ends near -2.5, as the
    reference's own learning filter's does on the same series."""
    T, ts = 5000, 2500
    h, y = _mu_regime_series()

    def rmse(hm, lo, hi):
        e = np.asarray(hm[lo:hi], dtype=np.float64) - h[lo:hi]
        return float(np.sqrt(np.mean(e * e)))

    res = {}
    for learn in (False, True):
        f = bpf.GpuBpf(4096, 0.98, 0.15, -1.0, 0.0, 5.0, 42)
        if learn:
            f.enable_mu_learning(1, 50, 0.1, 10.0, 0.667)
        hm = [f.step(float(v)).h_mean for v in y]
        res[learn] = (rmse(hm, 50, ts), rmse(hm, ts, T), f.get_mu())
        f.close()
    ref = None
    from oracle import refgpu
    if refgpu.available():
        g = refgpu.RefGpuFilter(4096, 0.98, 0.15, -1.0, 0.0, 5.0, seed=42)
        g.enable_mu_learning(1, 50, 0.1, 10.0, 0.667)
        hm_r, _ = g.run(y)
        ref = (rmse(hm_r, 50, ts), rmse(hm_r, ts, T), g.mu())
        g.close()
    print(f"\n  vanilla: P1 {res[False][0]:.4f} P2 {res[False][1]:.4f}; learning: P1 {res[True][0]:.4f} "
          f"P2 {res[True][1]:.4f} mu {res[True][2]:+.4f}; reference learning: {ref}")
    assert res[True][1] < res[False][1] - 0.05, res
    assert abs(res[True][2] - (-2.5)) < 0.5, res
    if ref is not None:                      # measured: mu -2.787 vs -2.791, phase-2 RMSE 0.4622 vs 0.4623
        assert abs(res[True][2] - ref[2]) < 0.1, (res, ref)
        assert abs(res[True][1] - ref[1]) < 0.02, (res, ref)


def test_rho_regime_learning_with_reference(bpf):
    """The reference's rho-regime test (smc2/test_mu_learning.cu:468-525, its first seed): rho falls
    from 0.98 to 0.90 at t = 2500 (mu -1.0, sigma_z 0.15, nu_obs 5, N = 4096, T = 5000); mu and rho
    learning from (mu, rho) = (-1.0, 0.98), this build against the reference's own learning filter
    on the same series: learnt rho, mu and phase-2 RMSE."""
    T, ts = 5000, 2500
    h, y = _mu_regime_series(rho2=0.90)

    def rmse(hm):
        e = np.asarray(hm[ts:T], dtype=np.float64) - h[ts:T]
        return float(np.sqrt(np.mean(e * e)))

    f = bpf.GpuBpf(4096, 0.98, 0.15, -1.0, 0.0, 5.0, 42)
    f.enable_mu_learning(1, 50, 0.1, 10.0, 0.667)
    f.enable_rho_learning(True)
    hm = [f.step(float(v)).h_mean for v in y]
    ours = (rmse(hm), f.get_rho(), f.get_mu())
    f.close()
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("oracle/_ref not built")
    g = refgpu.RefGpuFilter(4096, 0.98, 0.15, -1.0, 0.0, 5.0, seed=42)
    g.enable_mu_learning(1, 50, 0.1, 10.0, 0.667)
    g.enable_rho_learning(True)
    hm_r, _ = g.run(y)
    ref = (rmse(hm_r), g.rho_value(), g.mu())
    g.close()
    print(f"\n  mu+rho learning, phase-2 RMSE / rho / mu: ours {ours}, reference {ref}")
    assert abs(ours[0] - ref[0]) < 0.02, (ours, ref)
    assert abs(ours[1] - ref[1]) < 0.02, (ours, ref)
    assert abs(ours[2] - ref[2]) < 0.1, (ours, ref)
