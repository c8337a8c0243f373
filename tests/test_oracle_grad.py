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


@pytest.mark.parametrize("nu,nu_state", [(0.0, 0.0), (5.0, 0.0), (5.0, 5.0)])
def test_forward_and_reverse_mode_agree(orc, nu, nu_state):
    anc, y = _case()
    l0, g0, d0 = orc.grad_f64(256, *THETA, y, anc, seed=7, nu_obs=nu, mode=0, nu_state=nu_state)
    l1, g1, d1 = orc.grad_f64(256, *THETA, y, anc, seed=7, nu_obs=nu, mode=1, nu_state=nu_state)
    assert abs(l0 - l1) <= 1e-10 * abs(l0)
    np.testing.assert_allclose(g0, g1, rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(d0, d1, rtol=0, atol=1e-11)


@pytest.mark.parametrize("nu,nu_state", [(0.0, 0.0), (5.0, 0.0), (0.0, 4.0)])
def test_gradient_matches_central_differences(orc, nu, nu_state):
    anc, y = _case(N=300, T=40, seed=3)
    _, g, _ = orc.grad_f64(300, *THETA, y, anc, seed=11, nu_obs=nu, mode=1, nu_state=nu_state)
    th = np.array(THETA)
    for k in range(3):
        d = 1e-5 * abs(th[k])
        tp, tm = th.copy(), th.copy()
        tp[k] += d
        tm[k] -= d
        lp = orc.grad_f64(300, *tp, y, anc, seed=11, nu_obs=nu, mode=0, nu_state=nu_state)[0]
        lm = orc.grad_f64(300, *tm, y, anc, seed=11, nu_obs=nu, mode=0, nu_state=nu_state)[0]
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


def test_tstate_noise_distribution(orc):
    """Student-t state noise: z * sqrt(nu / chi2_k), k = round(nu). Sample moments of the oracle's
    counter-based draws against t(5): mean 0, variance nu/(nu-2) = 5/3 (reference test
    tests/test_icdf_diag.cu:251-253 expects std 1.291), and chi2 draws with k = 4 dof have mean 4."""
    L = orc.lib()
    n = 40000
    z = np.array([L.orc_icdf_f64(L.orc_uniform(L.orc_pcg32_draw_jump(42, i, 3))) for i in range(n)])
    sc = np.array([L.orc_tstate_scale(42, i, 3, 5, 5.0) for i in range(n)])
    e = z * sc
    assert abs(e.mean()) < 0.03
    assert abs(e.std() - math.sqrt(5.0 / 3.0)) < 0.04
    chi2 = 4.0 / np.array([L.orc_tstate_scale(7, i, 1, 4, 4.0) for i in range(n)]) ** 2
    assert abs(chi2.mean() - 4.0) < 0.06 and abs(chi2.var() - 8.0) < 0.5
