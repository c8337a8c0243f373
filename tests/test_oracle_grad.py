"""CPU tests of the oracle's gradient (oracle/bpf_oracle.c orc_grad_f64).

The oracle's two modes (forward-mode tangents, reverse-mode adjoint) are pinned
against each other, against central finite differences of the oracle's own
FP64 log-likelihood under common random numbers with the ancestors held
fixed, and against torch autograd of an independent FP64 restatement of the
same loss (the estimator of the reference's tests/diff_bpf.py:186-237: detached
resampling indices, values keep their gradient)."""
from __future__ import annotations

import math

import numpy as np
import pytest


def _case(N=256, T=30, seed=0):
    rng = np.random.default_rng(seed)
    anc = np.sort(rng.integers(0, N, (T, N)), axis=1).astype(np.int32)
    y = (rng.standard_normal(T) * 0.7).astype(np.float32)
    return anc, y


THETA = (-0.8, 0.95, 0.25)


@pytest.mark.parametrize("nu", [0.0, 5.0])
def test_forward_and_reverse_mode_agree(orc, nu):
    anc, y = _case()
    l0, g0, d0 = orc.grad_f64(256, *THETA, y, anc, seed=7, nu_obs=nu, mode=0)
    l1, g1, d1 = orc.grad_f64(256, *THETA, y, anc, seed=7, nu_obs=nu, mode=1)
    assert abs(l0 - l1) <= 1e-10 * abs(l0)
    np.testing.assert_allclose(g0, g1, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(d0, d1, rtol=0, atol=1e-11)


@pytest.mark.parametrize("nu", [0.0, 5.0])
def test_gradient_matches_central_differences(orc, nu):
    anc, y = _case(N=300, T=40, seed=3)
    _, g, _ = orc.grad_f64(300, *THETA, y, anc, seed=11, nu_obs=nu, mode=1)
    th = np.array(THETA)
    for k in range(3):
        d = 1e-5 * abs(th[k])
        tp, tm = th.copy(), th.copy()
        tp[k] += d
        tm[k] -= d
        lp = orc.grad_f64(300, *tp, y, anc, seed=11, nu_obs=nu, mode=0)[0]
        lm = orc.grad_f64(300, *tm, y, anc, seed=11, nu_obs=nu, mode=0)[0]
        fd = (lp - lm) / (2 * d)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_gradient_matches_torch_autograd(orc):
    torch = pytest.importorskip("torch")
    N, T, seed = 128, 25, 5
    anc, y = _case(N=N, T=T, seed=9)
    L = orc.lib()
    # the oracle's noise: slot i, draw t (draw 0 = initial particles)
    eps = np.array([[L.orc_icdf_f64(L.orc_uniform(L.orc_pcg32_draw_jump(seed, i, t))) for i in range(N)]
                    for t in range(T)])
    th = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    mu, rho, sig = th[0], th[1], th[2]
    e = torch.tensor(eps, dtype=torch.float64)
    yt = torch.tensor(y, dtype=torch.float64)
    h = mu + sig / torch.sqrt(1.0 - rho * rho) * e[0]
    loss = torch.zeros((), dtype=torch.float64)
    for t in range(T):
        if t > 0:
            h = mu + rho * (h[torch.as_tensor(anc[t - 1], dtype=torch.long)] - mu) + sig * e[t]
        lw = -0.5 * math.log(2 * math.pi) - 0.5 * h - 0.5 * yt[t] ** 2 * torch.exp(-h)
        loss = loss + torch.logsumexp(lw, 0) - math.log(N)
    loss.backward()
    ll, g, _ = orc.grad_f64(N, *THETA, y, anc, seed=seed, mode=1)
    assert abs(ll - loss.item()) <= 1e-10 * abs(ll)
    np.testing.assert_allclose(g, th.grad.numpy(), rtol=1e-9, atol=1e-10)
