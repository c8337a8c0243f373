"""The reference's own GPU filter, run on the same GPU, pins the oracle and the CUDA path.

oracle/_ref/librefgpu.so is the reference's PTX edition (gpu_bpf/gpu_bpf_ptx_full.cu with
ptx_assembly/bpf_kernels_full.ptx, comments stripped of non-ASCII bytes and the target set to
sm_100a) built by oracle/build_ref.py; the tests skip when it was not built.

  PCG32 states after create and after T ticks   bit-exact vs (s_0, inc) of the oracle and the
  (PTX :74-157)                                 counter-based jump s_t = A^t s_0 + B_t inc
  initial particles (PTX :103-218)              <= 1e-5 abs vs the oracle's FP32 restatement (the
                                                PTX uses approximate MUFU division / log / sqrt);
                                                the CUDA path's inverse CDF (Giles) within the
                                                FP32 Acklam error bound + 2e-6, times std_stat
  lock-step ticks: every tick recomputed by     propagation <= 1e-5 abs; weights <= 2e-5 rel;
  the oracle from the reference's own previous  h_mean <= 1e-5 abs; loglik <= 2e-5 rel; ancestors
  particles (gpu_bpf_ptx_full.cu:550-748)       equal except near-ties of the FP32 CDF (thrust's
                                                scan order, div.approx targets): <= 1% of N, each
                                                an adjacent parent
  whole runs, reference vs CUDA path            first tick loglik <= 1e-4 rel; mean |h_mean diff|
  (config 1: N=4096, T=1000, always resample)   <= 0.03 over the run; total loglik within 2.0 nats
                                                (independent Monte Carlo error once the runs part)
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0
PCG_A = 6364136223846793005
M64 = (1 << 64) - 1


@pytest.fixture(scope="module")
def ref():
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("oracle/_ref not built (the reference tree was absent at build time)")
    refgpu.lib()
    return refgpu


def _series(T, seed=42):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(ys, dtype=np.float32)


def _jump(t):
    a, b, cm, cp = 1, 0, PCG_A, 1
    while t:
        if t & 1:
            a, b = (a * cm) & M64, (b * cm + cp) & M64
        cp, cm = ((cm + 1) * cp) & M64, (cm * cm) & M64
        t >>= 1
    return a, b


def _init_states(orc, seed, n):
    s0 = np.zeros(n, dtype=np.uint64)
    inc = np.zeros(n, dtype=np.uint64)
    for i in range(n):
        s0[i], inc[i] = orc.pcg32_init(seed, i)
    return s0, inc


def _states_at(s0, inc, t):
    a, b = _jump(t)
    with np.errstate(over="ignore"):
        return s0 * np.uint64(a) + inc * np.uint64(b)


def test_reference_pcg_states_match_counter_jump(ref, orc):
    N, seed, T = 4097, 42, 7
    f = ref.RefGpuFilter(N, RHO, SIG, MU, seed=seed, ess_threshold=0.5)
    s0, inc = _init_states(orc, seed, N)
    r = f.rng()
    np.testing.assert_array_equal(r[:, 1], inc)
    np.testing.assert_array_equal(r[:, 0], _states_at(s0, inc, 1))      # draw 0 fed the initial particles
    np.testing.assert_array_equal(r, orc.ref_init(N, RHO, SIG, MU, seed)[0])
    f.run(_series(T))
    r = f.rng()
    assert f.timestep == T
    np.testing.assert_array_equal(r[:, 0], _states_at(s0, inc, T))      # ticks 1..T-1 drew once each
    np.testing.assert_array_equal(r[:, 1], inc)
    f.close()


def test_reference_initial_particles(ref, orc, bpf):
    N, seed = 4097, 42
    f = ref.RefGpuFilter(N, RHO, SIG, MU, seed=seed)
    h0 = f.particles()
    f.close()
    L = orc.lib()
    _, h_orc = orc.ref_init(N, RHO, SIG, MU, seed)
    err = np.abs(h0.astype(np.float64) - h_orc)
    assert err.max() <= 1e-5, err.max()
    std = math.sqrt(SIG * SIG / max(1.0 - RHO * RHO, 1e-6))
    u = np.array([L.orc_uniform(orc.pcg32_draw(seed, i, 0)) for i in range(N)], dtype=np.float32)
    z32 = np.array([L.orc_acklam_f32(float(v)) for v in u], dtype=np.float64)
    z64 = np.array([L.orc_icdf_f64(float(v)) for v in u])
    # the CUDA path: Giles' erfinv (|err| < 1e-6) against the reference's FP32 Acklam
    g = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, seed)
    ours = np.frombuffer(g.get_particles(), dtype=np.float32).astype(np.float64)
    g.close()
    bound = (np.abs(z32 - z64).max() + 2e-6) * std + 1e-6
    d = np.abs(ours - h0)
    assert d.max() <= bound, (d.max(), bound)


def test_reference_lockstep_ticks(ref, orc):
    N, seed, T = 4096, 42, 40
    y = _series(T)
    f = ref.RefGpuFilter(N, RHO, SIG, MU, seed=seed, ess_threshold=0.0)
    u23 = orc.host_u23_stream(seed, T)
    h_prev = f.particles()
    rng = np.ascontiguousarray(f.rng())
    worst = {"prop": 0.0, "w": 0.0, "hm": 0.0, "ll": 0.0, "anc": 0}
    for t in range(T):
        hm_r, ll_r = f.run(y[t:t + 1])
        pre, w, post = f.pre_resample_particles(), f.weights(), f.particles()
        # propagation from the reference's own previous particles and PCG32 states
        h_o, _, _, _, _ = orc.ref_tick(rng, h_prev, RHO, SIG, MU, y[t], propagate=t > 0)
        if t == 0:
            np.testing.assert_array_equal(pre, h_prev)
        e = float(np.abs(pre.astype(np.float64) - h_o).max())
        assert e <= 1e-5, (t, e)
        worst["prop"] = max(worst["prop"], e)
        # weights, mean and log-likelihood from the reference's propagated particles
        scratch = np.zeros((N, 2), dtype=np.uint64)
        _, w_o, hm_o, ll_o, _ = orc.ref_tick(scratch, pre, RHO, SIG, MU, y[t], propagate=False)
        ew = float(np.max(np.abs(w.astype(np.float64) - w_o) / np.maximum(w_o, 1e-30)))
        assert ew <= 2e-5, (t, ew)
        assert abs(hm_r[0] - hm_o) <= 1e-5 * max(1.0, abs(hm_o)), (t, hm_r[0], hm_o)
        assert abs(ll_r[0] - ll_o) <= 2e-5 * max(1.0, abs(ll_o)), (t, ll_r[0], ll_o)
        worst["w"] = max(worst["w"], ew)
        worst["hm"] = max(worst["hm"], abs(float(hm_r[0]) - hm_o))
        worst["ll"] = max(worst["ll"], abs(float(ll_r[0]) - ll_o))
        # systematic resampling of the reference's own weights with the host stream's U
        u = np.float32(np.float32(u23[t]) * np.float32(1.0 / 8388608.0)) / np.float32(N)
        anc = orc.ref_resample(w, float(u))
        bad = np.nonzero(post != pre[anc])[0]
        assert len(bad) <= N // 100, (t, len(bad))
        for i in bad:
            j = anc[i]
            near = pre[max(j - 2, 0):j + 3]
            assert post[i] in near, (t, i, j)
        worst["anc"] = max(worst["anc"], len(bad))
        h_prev = post
        rng = np.ascontiguousarray(f.rng())
    assert f.resample_count == T
    f.close()
    print("lock-step worst:", worst)


def test_reference_and_cuda_path_config1(ref, bpf, orc):
    N, seed, T = 4096, 42, 1000
    y = _series(T)
    f = ref.RefGpuFilter(N, RHO, SIG, MU, seed=seed, ess_threshold=0.0)
    hm_r, ll_r = f.run(y)
    f.close()
    g = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, seed, ess_threshold=0.0)
    recs = g.step_many(y.tolist(), records=True)
    g.close()
    hm_o = np.array([r.h_mean for r in recs], dtype=np.float64)
    ll_o = np.array([r.dloglik for r in recs], dtype=np.float64)
    assert abs(ll_r[0] - ll_o[0]) <= 1e-4 * max(1.0, abs(ll_o[0])), (ll_r[0], ll_o[0])
    dh = float(np.mean(np.abs(hm_r.astype(np.float64) - hm_o)))
    dll = float(np.sum(ll_r.astype(np.float64)) - np.sum(ll_o))
    assert dh <= 0.03, dh
    assert abs(dll) <= 2.0, dll
    print(f"config 1: mean |h_mean diff| {dh:.4f}, total loglik reference {np.sum(ll_r.astype(np.float64)):.4f} "
          f"ours {np.sum(ll_o):.4f}")
