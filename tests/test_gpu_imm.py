"""GPU tests of resumable batched stepping and of the IMM entry points (gpu_imm_*).

  batch stepped in pieces vs one run     loglik, per-tick increments and means bit-identical
  IMM vs the reference's recursion       model probabilities, mixed mean and log Z within 1e-6
  (gpu_bpf/gpu_bpf.cu:1023-1078) fed     (float outputs) of a host restatement fed the same
  the models' own increments             per-model increments
  IMM vs independent plain filters       <= 5e-3 absolute on the probabilities (the batched
                                         increments differ from the plain ones by summation order)
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODELS = [
    {"rho": 0.97, "sigma_z": 0.15, "mu": -1.0},
    {"rho": 0.90, "sigma_z": 0.30, "mu": -0.5},
    {"rho": 0.99, "sigma_z": 0.05, "mu": -1.5, "nu_obs": 5.0},
    {"rho": 0.95, "sigma_z": 0.20, "mu": -1.0, "nu_state": 5.0},
]


def _series(T, seed=42, rho=0.97, sig=0.15, mu=-1.0):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def _lse(x):
    m = np.max(x)
    return m + math.log(np.sum(np.exp(x - m)))


def _imm_host(dll, hm, K, log_T):
    """The reference's IMM recursion (gpu_bpf/gpu_bpf.cu:1023-1078) on given increments."""
    log_pi = np.full(K, -math.log(K))
    out = []
    for t in range(dll.shape[1]):
        pred = np.array([_lse(log_T[:, k] + log_pi) for k in range(K)])
        joint = pred + dll[:, t]
        lz = _lse(joint)
        log_pi = joint - lz
        pi = np.exp(log_pi)
        out.append((pi.copy(), float(np.sum(pi * hm[:, t])), lz))
    return out


@pytest.mark.parametrize("thr", [0.0, 0.5])
def test_batch_steps_equal_one_run(bpf, thr):
    import torch
    from gpubpf import configs
    fl = configs.batch_thetas(12)
    for i, f in enumerate(fl):
        f["n_particles"] = [700, 3000, 9000, 16384][i % 4]
    y = _series(47)
    T, B = len(y), len(fl)
    y_d = torch.tensor(y, device="cuda")
    b = bpf.GpuBpfBatch(fl, ess_threshold=thr)
    ll = torch.zeros(B, dtype=torch.float64, device="cuda")
    dll = torch.zeros(B * T, dtype=torch.float64, device="cuda")
    hm = torch.zeros(B * T, dtype=torch.float32, device="cuda")
    b.run_device(y_d.data_ptr(), T, ll.data_ptr(), dll.data_ptr(), hm.data_ptr())
    torch.cuda.synchronize()
    ll_full, dll_full, hm_full = ll.cpu().numpy(), dll.cpu().numpy().reshape(B, T), hm.cpu().numpy().reshape(B, T)
    for rep in range(2):                                  # the second pass starts again after reset
        # runs of equal lengths at moving pointers take the direct launch, new lengths a new graph
        pieces, t0 = [1, 1, 1, 5, 13, 1, 1, 24], 0
        dll_s = np.zeros((B, T))
        hm_s = np.zeros((B, T), dtype=np.float32)
        for n in pieces:
            d = torch.zeros(B * n, dtype=torch.float64, device="cuda")
            h = torch.zeros(B * n, dtype=torch.float32, device="cuda")
            b.step_device(y_d[t0:].data_ptr(), n, d.data_ptr(), h.data_ptr())
            torch.cuda.synchronize()
            dll_s[:, t0:t0 + n] = d.cpu().numpy().reshape(B, n)
            hm_s[:, t0:t0 + n] = h.cpu().numpy().reshape(B, n)
            t0 += n
        assert t0 == T and b.tick == T
        np.testing.assert_array_equal(dll_s, dll_full)
        np.testing.assert_array_equal(hm_s, hm_full)
        for i in range(B):                                # the kernel's running FP64 sum, same order
            acc = 0.0
            for t in range(T):
                acc += float(dll_s[i, t])
            assert acc == ll_full[i]
        b.reset()
    b.close()


def test_imm_matches_reference_recursion(bpf):
    import torch
    K, N, T, seed = len(MODELS), 3000, 60, 11
    y = _series(T)
    imm = bpf.Imm(MODELS, N, seed=seed)
    res = [imm.step(float(v)) for v in y]
    probs = np.array(imm.probs())
    st = imm.state
    log_T = np.array([st.log_T[i] for i in range(K * K)]).reshape(K, K)
    assert st.timestep == T
    imm.close()
    # the same K filters as one batched run (seed + 7919 k, ESS threshold 0.5)
    fl = [dict(m, n_particles=N, seed=seed + 7919 * k) for k, m in enumerate(MODELS)]
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(K, dtype=torch.float64, device="cuda")
    dll = torch.zeros(K * T, dtype=torch.float64, device="cuda")
    hm = torch.zeros(K * T, dtype=torch.float32, device="cuda")
    b.run_device(y_d.data_ptr(), T, ll.data_ptr(), dll.data_ptr(), hm.data_ptr())
    torch.cuda.synchronize()
    b.close()
    ref = _imm_host(dll.cpu().numpy().reshape(K, T), hm.cpu().numpy().reshape(K, T).astype(np.float64), K, log_T)
    for t, (r, (pi, hmix, lz)) in enumerate(zip(res, ref)):
        assert abs(r.h_mean - hmix) <= 1e-6 * max(1.0, abs(hmix)), t
        assert abs(r.log_lik - lz) <= 1e-6 * max(1.0, abs(lz)), t
        assert r.best_model == int(np.argmax(pi))
        assert abs(r.best_prob - pi.max()) <= 1e-6
    np.testing.assert_allclose(probs, ref[-1][0], rtol=1e-6, atol=1e-7)
    # against K independent plain filters (the reference's own arrangement)
    dll_p = np.zeros((K, T))
    hm_p = np.zeros((K, T))
    for k, m in enumerate(MODELS):
        f = bpf.GpuBpf(N, m["rho"], m["sigma_z"], m["mu"], m.get("nu_state", 0.0), m.get("nu_obs", 0.0),
                       seed + 7919 * k)
        for t in range(T):
            f.step(float(y[t]))
            rec = f.get_record()
            dll_p[k, t], hm_p[k, t] = rec.dloglik, rec.h_mean
        f.close()
    ref_p = _imm_host(dll_p, hm_p, K, log_T)
    np.testing.assert_allclose(probs, ref_p[-1][0], atol=5e-3)


def test_imm_plain_filter_path_and_transition_matrix(bpf):
    """More than 16384 particles per model: the models run as plain filters."""
    K, N, T, seed = 2, 20000, 12, 5
    tm = [0.9, 0.1, 0.2, 0.8]
    y = _series(T)
    imm = bpf.Imm(MODELS[:K], N, transition_matrix=tm, seed=seed)
    assert imm.state.filters
    res = [imm.step(float(v)) for v in y]
    imm.close()
    dll_p = np.zeros((K, T))
    hm_p = np.zeros((K, T))
    for k, m in enumerate(MODELS[:K]):
        f = bpf.GpuBpf(N, m["rho"], m["sigma_z"], m["mu"], 0.0, 0.0, seed + 7919 * k)
        for t in range(T):
            f.step(float(y[t]))
            rec = f.get_record()
            dll_p[k, t], hm_p[k, t] = rec.dloglik, rec.h_mean
        f.close()
    log_T = np.log(np.array(tm, dtype=np.float64).reshape(K, K).astype(np.float32).astype(np.float64))
    ref = _imm_host(dll_p, hm_p, K, log_T)
    for r, (pi, hmix, lz) in zip(res, ref):
        assert abs(r.h_mean - hmix) <= 1e-6 * max(1.0, abs(hmix))
        assert abs(r.log_lik - lz) <= 1e-6 * max(1.0, abs(lz))


def test_imm_finds_the_generating_model(bpf):
    """With sticky switching the model that generated the series carries most of the
    probability over the second half of the run (model probabilities are filtered per tick,
    so single ticks may favour another model)."""
    grid = bpf.build_grid([0.97], [0.05, 0.2, 0.6], [-1.0])
    y = _series(800, seed=3, rho=0.97, sig=0.2, mu=-1.0)
    K = len(grid)
    tm = [0.999 if i == j else 0.0005 for i in range(K) for j in range(K)]
    imm = bpf.Imm(grid, 4096, transition_matrix=tm, seed=1)
    acc = np.zeros(K)
    for t, v in enumerate(y):
        imm.step(float(v))
        p = np.array(imm.probs())
        assert abs(p.sum() - 1.0) < 1e-5
        if t >= 400:
            acc += p
    imm.close()
    assert int(np.argmax(acc)) == 1, acc
