"""GPU tests of the batched autograd face (BpfBatchLoglik / bpf_batch_loglik over gpu_bpf_batch_grad_run).

  loglik[B] and theta.grad                      bit-identical to one gpu_bpf_batch_grad_run of a
                                                batch built with the same theta (the backward only
                                                scales the gradient of that run)
  a second call with new theta                  equals a fresh batch at the new theta (the cached
                                                batch takes the new parameters)
  against plain gradient tapes                  loglik <= 1e-6 relative, gradient <= 1e-4 of its
                                                largest component (the batched gradient's bound)
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = [700, 4096, 9000]
SEEDS = [11, 12, 13]


def _series(T, seed=42):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, 0.97, 0.2, -1.0, seed)
    return np.asarray(ys, dtype=np.float32)


def _direct(bpf, theta, y):
    import torch
    fl = [{"mu": m, "rho": r, "sigma_z": s, "n_particles": n, "seed": q} for (m, r, s), n, q in zip(theta, N, SEEDS)]
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.0)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(len(N), dtype=torch.float64, device="cuda")
    g = torch.zeros(len(N) * 3, dtype=torch.float64, device="cuda")
    b.grad_run(y_d.data_ptr(), len(y), ll.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()
    b.close()
    return ll.cpu().numpy(), g.cpu().numpy().reshape(-1, 3)


def test_batch_autograd_matches_grad_run(bpf):
    import torch
    y = _series(60)
    th0 = [(-1.0, 0.97, 0.2), (-0.6, 0.92, 0.3), (-1.3, 0.98, 0.12)]
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    ll = bpf.bpf_batch_loglik(theta, torch.tensor(y, device="cuda"), N, SEEDS)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64, device="cuda")
    (w * ll).sum().backward()
    ll_d, g_d = _direct(bpf, th0, y)
    np.testing.assert_array_equal(ll.detach().cpu().numpy(), ll_d)
    np.testing.assert_array_equal(theta.grad.numpy(), w.cpu().numpy()[:, None] * g_d)


def test_batch_autograd_new_theta_and_plain_tapes(bpf):
    import torch
    y = _series(50, seed=3)
    th_a = [(-1.0, 0.97, 0.2), (-0.6, 0.92, 0.3), (-1.3, 0.98, 0.12)]
    th_b = [(-0.9, 0.95, 0.25), (-0.7, 0.9, 0.35), (-1.1, 0.97, 0.15)]
    y_d = torch.tensor(y, device="cuda")
    bpf.bpf_batch_loglik(torch.tensor(th_a, dtype=torch.float64), y_d, N, SEEDS)
    theta = torch.tensor(th_b, dtype=torch.float64, requires_grad=True)
    ll = bpf.bpf_batch_loglik(theta, y_d, N, SEEDS)
    ll.sum().backward()
    ll_d, g_d = _direct(bpf, th_b, y)
    np.testing.assert_array_equal(ll.detach().cpu().numpy(), ll_d)
    np.testing.assert_array_equal(theta.grad.numpy(), g_d)
    for i, (m, r, s) in enumerate(th_b):
        tape = bpf.GradTape(N[i], len(y), checkpoint_every=8)
        pll = tape.forward((m, r, s), y_d, seed=SEEDS[i]).item()
        pg = tape.backward().cpu().numpy()
        tape.close()
        assert abs(ll_d[i] - pll) <= 1e-6 * max(1.0, abs(pll))
        assert np.max(np.abs(g_d[i] - pg)) <= 1e-4 * np.max(np.abs(pg))
