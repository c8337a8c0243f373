"""GPU tests of the auxiliary particle filter (gpu_apf_*; reference gpu_bpf_ptx_full.cu:990-1190).

  APF vs the FP64 oracle on the device's       per tick: APF increment, the reference's log mean
  ancestors of both stages (orc_apf_f64)       second-stage weight and h_mean <= 2e-4 absolute;
  (Gaussian, Student-t obs, Student-t state)   total increment <= 1e-4 relative
  tick 0                                       equals a bootstrap filter's tick 0 bit for bit
  gpu_apf_step_many (graphs) vs gpu_apf_step    records bit-identical
  gpu_apf_run_rmse                              equals the RMSE of the step_many means
  vs the reference's own APF on the same GPU   statistical (its noise is cuRAND XORWOW): mean
  (skipped when oracle/_ref is not built)      |h_mean diff| <= 0.03 over 1000 ticks, RMSE to the
                                               true h within 0.02, sum of log_lik within 3 nats
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def _series(T, seed=42):
    from gpubpf import dgp
    h, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(h), np.asarray(ys, dtype=np.float32)


@pytest.mark.parametrize("nu_obs,nu_state", [(0.0, 0.0), (5.0, 0.0), (0.0, 5.0)])
def test_apf_matches_fp64_oracle_on_device_ancestors(bpf, orc, nu_obs, nu_state):
    N, T, seed = 4096, 60, 11
    _, y = _series(T)
    f = bpf.GpuApf(N, RHO, SIG, MU, nu_state, nu_obs, seed)
    f.record_ancestors(True)
    anc1 = np.zeros((T, N), dtype=np.int32)
    anc2 = np.zeros((T, N), dtype=np.int32)
    recs = []
    for t in range(T):
        r = f.step(float(y[t]))
        rec = f.get_record()
        assert rec.tick == t and rec.resampled == 1
        assert r.log_lik == np.float32(rec.loglik_ref)
        a1, a2 = f.get_ancestors()
        anc1[t] = np.frombuffer(a1, dtype=np.int32)
        anc2[t] = np.frombuffer(a2, dtype=np.int32)
        for a in (anc2[t],) if t == 0 else (anc1[t], anc2[t]):
            assert a.min() >= 0 and a.max() < N and np.all(np.diff(a) >= 0)     # systematic: monotone
        recs.append(rec)
    total = f.get_loglik_total()
    assert f.state.timestep == T
    f.close()
    o = orc.apf_f64(N, RHO, SIG, MU, y, seed=seed, nu_obs=nu_obs, nu_state=nu_state, anc1=anc1, anc2=anc2)
    dll = np.array([r.dloglik for r in recs])
    llr = np.array([r.loglik_ref for r in recs])
    hm = np.array([r.h_mean for r in recs])
    np.testing.assert_allclose(dll, o["dll"], atol=2e-4, rtol=0)
    np.testing.assert_allclose(llr, o["ll_ref"], atol=2e-4, rtol=0)
    np.testing.assert_allclose(hm, o["hmean"], atol=2e-4, rtol=0)
    assert abs(dll.sum() - o["dll"].sum()) <= 1e-4 * abs(o["dll"].sum())
    assert abs(total - dll.sum()) <= 1e-9 * abs(total)


def test_apf_tick0_is_a_bootstrap_tick(bpf):
    N, seed = 5000, 3
    _, y = _series(4)
    a = bpf.GpuApf(N, RHO, SIG, MU, 0.0, 0.0, seed)
    b = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, seed, ess_threshold=0.0)
    a.step(float(y[0]))
    b.step(float(y[0]))
    ra, rb = a.get_record(), b.get_record()
    assert ra.dloglik == rb.dloglik and ra.h_mean == rb.h_mean and ra.ess == rb.ess
    assert bytes(a.get_particles()) == bytes(b.get_particles())
    a.close()
    b.close()


def test_apf_step_many_equals_steps(bpf):
    N, T, seed = 3000, 150, 5
    _, y = _series(T)
    a = bpf.GpuApf(N, RHO, SIG, MU, 0.0, 5.0, seed)
    ra = a.step_many(y.tolist(), records=True)          # tick 0 direct, then 64-tick graphs + remainder
    b = bpf.GpuApf(N, RHO, SIG, MU, 0.0, 5.0, seed)
    rb = []
    for v in y:
        b.step(float(v))
        rb.append(b.get_record())
    for x, z in zip(ra, rb):
        assert (x.dloglik, x.loglik_ref, x.h_mean, x.ess, x.tick) == (z.dloglik, z.loglik_ref, z.h_mean, z.ess, z.tick)
    assert a.get_loglik_total() == b.get_loglik_total()
    assert bytes(a.get_particles()) == bytes(b.get_particles())
    a.close()
    b.close()


def test_apf_run_rmse(bpf):
    N, T, seed = 4096, 400, 42
    h, y = _series(T)
    v = bpf.apf_run_rmse(y.astype(np.float64).tolist(), h.tolist(), N, RHO, SIG, MU, 0.0, 0.0, seed)
    f = bpf.GpuApf(N, RHO, SIG, MU, 0.0, 0.0, seed)
    out = f.step_many(y.tolist())
    f.close()
    hm = np.array([r.h_mean for r in out], dtype=np.float64)
    expect = math.sqrt(np.mean((hm[100:] - h[100:]) ** 2))
    assert abs(v - expect) <= 1e-12 * expect
    assert 0.2 < v < 0.8


def test_apf_vs_reference_apf(bpf):
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("oracle/_ref not built")
    N, T, seed = 4096, 1000, 42
    h, y = _series(T)
    hm_r, ll_r = refgpu.apf_run(N, RHO, SIG, MU, y, seed=seed)
    f = bpf.GpuApf(N, RHO, SIG, MU, 0.0, 0.0, seed)
    out = f.step_many(y.tolist())
    f.close()
    hm = np.array([r.h_mean for r in out], dtype=np.float64)
    ll = np.array([r.log_lik for r in out], dtype=np.float64)
    dh = float(np.mean(np.abs(hm - hm_r)))
    rmse_o = math.sqrt(np.mean((hm[100:] - h[100:]) ** 2))
    rmse_r = math.sqrt(np.mean((hm_r[100:].astype(np.float64) - h[100:]) ** 2))
    dll = float(ll.sum() - ll_r.astype(np.float64).sum())
    print(f"APF vs reference APF: mean |h_mean diff| {dh:.4f}, RMSE ours {rmse_o:.4f} reference {rmse_r:.4f}, "
          f"sum log_lik ours {ll.sum():.4f} reference {ll_r.astype(np.float64).sum():.4f}")
    assert dh <= 0.03
    assert abs(rmse_o - rmse_r) <= 0.02
    assert abs(dll) <= 3.0
