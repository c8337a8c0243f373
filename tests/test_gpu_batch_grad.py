"""GPU tests of the batched gradient (gpu_bpf_batch_grad_run) through the C ABI.

A batched filter reproduces the plain filter's ancestors and particles bit for bit, and its
backward pass is the plain adjoint's arithmetic with sums in another order, so against a plain
gradient tape with the same (theta, N, seed):
  total log-likelihood   <= 1e-6 relative
  gradient               <= 1e-4 relative to the largest component
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FILTERS = [
    {"mu": -1.0, "rho": 0.97, "sigma_z": 0.15, "n_particles": 1, "seed": 3},
    {"mu": -0.5, "rho": 0.90, "sigma_z": 0.30, "n_particles": 100, "seed": 4},
    {"mu": -1.2, "rho": 0.99, "sigma_z": 0.10, "n_particles": 4096, "seed": 5},
    {"mu": -0.8, "rho": 0.95, "sigma_z": 0.25, "n_particles": 5000, "seed": 6},
    {"mu": -1.5, "rho": 0.85, "sigma_z": 0.40, "n_particles": 9000, "seed": 7},
    {"mu": -1.0, "rho": 0.97, "sigma_z": 0.20, "n_particles": 16384, "seed": 8},
]


def _series(T, seed=42):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, 0.97, 0.2, -1.0, seed)
    return np.asarray(ys, dtype=np.float32)


def _batch_grad(bpf, filters, y, threads=None):
    import torch
    b = bpf.GpuBpfBatch(filters, ess_threshold=0.0)
    if threads:
        for c, t in threads.items():
            b.set_threads(c, t)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(len(filters), dtype=torch.float64, device="cuda")
    g = torch.zeros(len(filters) * 3, dtype=torch.float64, device="cuda")
    b.grad_run(y_d.data_ptr(), len(y), ll.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()
    b.close()
    return ll.cpu().numpy(), g.cpu().numpy().reshape(-1, 3)


def _plain_grad(bpf, f, y):
    import torch
    tape = bpf.GradTape(f["n_particles"], len(y), checkpoint_every=8)
    ll = tape.forward((f["mu"], f["rho"], f["sigma_z"]), torch.tensor(y, device="cuda"), seed=f["seed"],
                      nu_obs=f.get("nu_obs", 0.0)).item()
    g = tape.backward().cpu().numpy()
    tape.close()
    return ll, g


def _check(bpf, filters, y, ll, g):
    for i, f in enumerate(filters):
        pll, pg = _plain_grad(bpf, f, y)
        assert abs(ll[i] - pll) <= 1e-6 * max(1.0, abs(pll)), (i, ll[i], pll)
        assert np.max(np.abs(g[i] - pg)) <= 1e-4 * np.max(np.abs(pg)), (i, g[i], pg)


def test_batch_grad_matches_plain_tapes(bpf):
    y = _series(60)
    ll, g = _batch_grad(bpf, FILTERS, y)
    _check(bpf, FILTERS, y, ll, g)


def test_batch_grad_student_t_and_segments(bpf):
    fl = [dict(f, nu_obs=5.0) for f in FILTERS[2:5]]
    y = _series(37, seed=3)                     # 37 ticks: last checkpoint segment is partial
    ll, g = _batch_grad(bpf, fl, y)
    _check(bpf, fl, y, ll, g)


def test_batch_grad_regime_series(bpf):
    from gpubpf import configs, dgp
    fl = configs.config5(6)
    _, ys = dgp.regime_series(300, period=100, seed=42)
    y = np.asarray(ys, dtype=np.float32)
    ll, g = _batch_grad(bpf, fl, y)
    assert np.all(np.isfinite(g))
    _check(bpf, fl[:3], y, ll, g)


def test_batch_grad_deterministic_and_shape_independent(bpf):
    y = _series(40)
    fl = FILTERS[1:]
    a = _batch_grad(bpf, fl, y)
    b = _batch_grad(bpf, fl, y)
    np.testing.assert_array_equal(a[1], b[1])
    c = _batch_grad(bpf, fl, y, threads={0: 64, 2: 512, 3: 1024, 4: 512})
    np.testing.assert_allclose(c[0], a[0], rtol=1e-9)
    np.testing.assert_allclose(c[1], a[1], rtol=1e-5, atol=1e-6 * np.max(np.abs(a[1])))


def test_batch_grad_requires_always_resample(bpf):
    import torch
    from gpubpf._lib import BpfError
    b = bpf.GpuBpfBatch(FILTERS[1:3], ess_threshold=0.5)
    y = torch.zeros(10, device="cuda")
    ll = torch.zeros(2, dtype=torch.float64, device="cuda")
    g = torch.zeros(6, dtype=torch.float64, device="cuda")
    with pytest.raises(BpfError) as ei:
        b.grad_run(y.data_ptr(), 10, ll.data_ptr(), g.data_ptr())
    assert ei.value.code == 4
    b.close()
