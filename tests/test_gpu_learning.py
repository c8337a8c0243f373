"""GPU tests of online mu / rho learning (gpu_bpf_enable_mu_learning and friends).

  score sums vs a host restatement      <= 1e-4 relative (FP32 particles and weights, FP64 sums)
  (PTX :1187-1227: sum W dlw, sum W dlw^2,
  sum W dlw dh, sum W dlw^2 dh^2)
  update rule vs a host restatement     <= 1e-5 relative on mu and rho (the reference's formulas,
  (gpu_bpf_ptx_full.cu:489-543)         fed the same sums)
  learning from a wrong mu              moves mu most of the way to the generating value
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
