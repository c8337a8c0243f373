"""GPU tests of the SMC^2 driver (gpu_bpf_smc2_*).

  no moves, no outer resampling     every theta-particle's inner log-likelihood and outer
                                    log-weight equal a batched run with its theta and seed, bit
                                    for bit (the inner filters are the resumable batch)
  same seed                         identical posterior (deterministic driver)
  synthetic data                    the posterior contracts around the generating theta
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(T, theta=(-1.0, 0.95, 0.25), seed=42):
    from gpubpf import dgp
    mu, rho, sig = theta
    _, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def test_smc2_without_moves_is_the_batched_filter(bpf):
    import torch
    M, N, T, seed = 40, 700, 50, 9
    y = _series(T)
    s = bpf.Smc2(M, N, T, seed=seed)
    s.set_moves(0, 0.0, 1.0)                     # never resample the theta-particles
    for v in y:
        assert s.update(float(v)) > 0
    th, lw, ll = s.particles()
    assert s.stats()["rejuvenations"] == 0
    s.close()
    np.testing.assert_array_equal(lw, ll)
    fl = [{"mu": float(th[j, 0]), "rho": float(th[j, 1]), "sigma_z": float(th[j, 2]), "n_particles": N,
           "seed": (seed & 0x3fffffff) + 1 + j} for j in range(M)]
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    out = torch.zeros(M, dtype=torch.float64, device="cuda")
    b.run_device(torch.tensor(y, device="cuda").data_ptr(), T, out.data_ptr())
    torch.cuda.synchronize()
    b.close()
    np.testing.assert_array_equal(ll, out.cpu().numpy())


def test_smc2_is_deterministic(bpf):
    y = _series(150, seed=5)
    res = []
    for _ in range(2):
        s = bpf.Smc2(64, 512, 150, seed=3)
        ess = [s.update(float(v)) for v in y]
        res.append((s.theta(), ess, s.stats()))
        s.close()
    np.testing.assert_array_equal(res[0][0][0], res[1][0][0])
    np.testing.assert_array_equal(res[0][0][1], res[1][0][1])
    assert res[0][1] == res[1][1] and res[0][2] == res[1][2]
    assert res[0][2]["rejuvenations"] > 0


def test_smc2_posterior_contracts_around_the_truth(bpf):
    truth = (-1.0, 0.95, 0.25)
    T = 600
    y = _series(T, truth, seed=11)
    s = bpf.Smc2(256, 512, T, seed=7)
    s.set_moves(2, 0.5, 1.0)
    for v in y:
        s.update(float(v))
    mean, sd = s.theta()
    st = s.stats()
    s.close()
    assert st["rejuvenations"] >= 3
    rate = st["accepted"] / max(1, st["proposed"])
    assert 0.02 < rate < 0.95, st
    assert abs(mean[0] - truth[0]) < 3 * sd[0] + 0.1, (mean, sd)
    assert sd[0] < 0.35                          # the N(-1, 0.5^2) prior on mu has contracted
    assert abs(mean[2] - truth[2]) < 3 * sd[2] + 0.05, (mean, sd)
    assert 0.85 < mean[1] < 0.995


@pytest.mark.parametrize("cp_rho", [0.0, 0.99])
def test_smc2_outer_loop_matches_host_restatement(bpf, cp_rho):
    """Every outer step of a real update sequence against the host restatement of the outer loop
    (oracle/smc2_outer.py, the reference's smc2_cuda_update outer step on this SV model) fed the
    device's inner log-likelihoods: the prior draws, each tick's outer ESS, whether it resamples,
    the outer ancestors, every proposal and acceptance flag bit for bit, and the outer log-weights
    exactly (within 1e-12)."""
    from oracle.smc2_outer import Smc2Outer
    M, N, T, seed = 48, 256, 120, 11
    y = _series(T, seed=6)
    s = bpf.Smc2(M, N, T, seed=seed)
    s.set_moves(1, 0.5, 1.0)
    if cp_rho > 0:
        s.set_cpmmh_rho(cp_rho)
    ref = Smc2Outer(M, seed)
    th, _, _ = s.particles()
    np.testing.assert_array_equal(th, ref.theta_f32())
    n_res = n_acc = 0
    for t, v in enumerate(y):
        ess = s.update(float(v))
        lu = s.last_update()
        ess_ref, res_ref = ref.observe(lu["dll"])
        assert res_ref == lu["resampled"], t
        if res_ref:
            n_res += 1
            assert ess == np.float32(M)
            assert list(lu["ancestors"]) == ref.resample(), t
            scored, cur = ref.propose()
            mv = s.last_move()
            np.testing.assert_array_equal(mv["theta_prop"], scored)
            np.testing.assert_array_equal(mv["theta_cur"], cur)
            flags = ref.accept(mv["loglik_prop"], mv["loglik_cur"])
            assert list(mv["accepted"]) == flags, t
            n_acc += sum(flags)
        else:
            assert ess == np.float32(ess_ref), t
        th, lw, _ = s.particles()
        np.testing.assert_array_equal(th, ref.theta_f32())
        assert np.max(np.abs(lw - np.asarray(ref.logw))) <= 1e-12
    st = s.stats()
    s.close()
    assert n_res >= 2 and st["rejuvenations"] == n_res and st["accepted"] == n_acc
