"""GPU tests of the gradient form through the C ABI.

Tolerances
  taped forward vs plain filter      bit-identical total log-likelihood (same kernels)
  tape children vs plain ancestors   bit-exact
  adjoint vs FP64 CPU oracle         <= 1e-4 relative to the largest component (oracle replays the
                                     tape's ancestors; FP32 particles and normals vs FP64)
  adjoint vs FP64 replay tangents    <= 1e-4 relative to the largest component
  adjoint vs central differences     <= 1e-3 relative to the largest component: 5-point central
                                     stencil, step 1e-3*|theta_k|, on the FP64 replay (common random
                                     numbers, ancestors replayed). The 3-point difference's O(h^2)
                                     error in rho is ~1e-2 relative at that step (L is strongly curved
                                     in rho near 1), so it is checked for mu and sigma only
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETA = (-0.8, 0.95, 0.25)


def _series(T, seed=42, theta=THETA):
    from gpubpf import dgp
    mu, rho, sig = theta
    _, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


def test_taped_forward_equals_plain_filter(bpf):
    import torch
    N, T = 5000, 120
    y = _series(T)
    tape = bpf.GradTape(N, T)
    ll = tape.forward(THETA, torch.tensor(y, device="cuda"), seed=42).item()
    f = bpf.GpuBpf(N, THETA[1], THETA[2], THETA[0], 0.0, 0.0, 42, ess_threshold=0.0)
    f.record_ancestors(True)
    for t in range(T):
        f.step(float(y[t]))
        res, a = f.get_ancestors()
        assert res == 1
        np.testing.assert_array_equal(tape.ancestors(t), np.frombuffer(a, dtype=np.int32), err_msg=f"tick {t}")
    ll_plain = f.get_record().loglik_total
    f.close()
    assert ll == ll_plain
    tape.close()


def test_children_of_degenerate_ticks(bpf):
    """Outlying observations concentrate the weight on a few parents: their child runs go
    through the warp-shared walk; the tape must still match the plain filter."""
    import torch
    N, T = 70001, 12
    y = _series(T)
    y[3] = 9.0
    y[7] = -12.0
    tape = bpf.GradTape(N, T, checkpoint_every=5)
    tape.forward(THETA, torch.tensor(y, device="cuda"), seed=9)
    f = bpf.GpuBpf(N, THETA[1], THETA[2], THETA[0], 0.0, 0.0, 9, ess_threshold=0.0)
    f.record_ancestors(True)
    most = 0
    for t in range(T):
        f.step(float(y[t]))
        _, a = f.get_ancestors()
        anc = np.frombuffer(a, dtype=np.int32)
        np.testing.assert_array_equal(tape.ancestors(t), anc)
        most = max(most, int(np.max(np.bincount(anc))))
    assert most > 32          # some parent's children went through the warp-shared walk
    f.close()
    g = tape.backward().cpu().numpy()
    rep = tape.replay(THETA).cpu().numpy()
    assert _rel(g, rep[1:]) <= 1e-4
    tape.close()


@pytest.mark.parametrize("nu", [0.0, 5.0])
def test_adjoint_matches_fp64_oracle(bpf, orc, nu):
    import torch
    N, T, seed = 4096, 150, 42
    y = _series(T)
    tape = bpf.GradTape(N, T, checkpoint_every=16)
    ll = tape.forward(THETA, torch.tensor(y, device="cuda"), seed=seed, nu_obs=nu).item()
    g = tape.backward().cpu().numpy()
    anc = np.stack([tape.ancestors(t) for t in range(T)])
    oll, og, _ = orc.grad_f64(N, *THETA, y, anc, seed=seed, nu_obs=nu, mode=1)
    assert abs(ll - oll) <= 1e-4 * abs(oll)
    assert _rel(g, og) <= 1e-4, (g, og)
    tape.close()


def test_adjoint_matches_replay_and_central_differences(bpf):
    import torch
    N, T = 1 << 16, 400
    y = _series(T)
    tape = bpf.GradTape(N, T)
    ll = tape.forward(THETA, torch.tensor(y, device="cuda"), seed=42).item()
    g = tape.backward().cpu().numpy()
    rep = tape.replay(THETA).cpu().numpy()
    assert abs(rep[0] - ll) <= 1e-5 * abs(ll)            # FP64 replay of the FP32 run
    assert _rel(g, rep[1:]) <= 1e-4
    fd = tape.fd_gradient(THETA, rel=1e-3, points=5)
    assert _rel(g, fd) <= 1e-3, (g, fd)
    fd3 = tape.fd_gradient(THETA, rel=1e-3, points=3)     # O(h^2): mu and sigma still agree closely
    assert abs(fd3[0] - g[0]) <= 1e-4 * abs(g).max() and abs(fd3[2] - g[2]) <= 1e-4 * abs(g).max()
    tape.close()


def test_backward_is_deterministic_and_checkpoint_independent(bpf):
    import torch
    N, T = 30000, 97
    y = torch.tensor(_series(T), device="cuda")
    grads = []
    for K in (1, 7, 16, 97):
        tape = bpf.GradTape(N, T, checkpoint_every=K)
        tape.forward(THETA, y, seed=5)
        grads.append(tape.backward().cpu().numpy())
        grads.append(tape.backward().cpu().numpy())
        tape.close()
    for gk in grads[1:]:
        np.testing.assert_array_equal(gk, grads[0])


def test_autograd_function(bpf):
    import torch
    N, T = 8192, 60
    y = torch.tensor(_series(T), device="cuda")
    theta = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    ll = bpf.bpf_loglik(theta, y, N, seed=3)
    (-ll).backward()
    tape = bpf.GradTape(N, T)
    tape.forward(THETA, y, seed=3)
    g = tape.backward().cpu()
    torch.testing.assert_close(theta.grad, -g, rtol=0, atol=0)
    # a second forward on the same tape invalidates the first graph's backward
    ll2 = bpf.bpf_loglik(theta, y, N, seed=3)
    bpf.bpf_loglik(theta, y, N, seed=4)
    with pytest.raises(RuntimeError):
        ll2.backward()
    tape.close()


def test_errors(bpf):
    import torch
    from gpubpf._lib import BpfError
    tape = bpf.GradTape(1000, 10)
    with pytest.raises(BpfError):
        tape.backward()                                   # no forward yet
    y = torch.zeros(10, device="cuda")
    lib = bpf.load()
    rc = lib.gpu_bpf_grad_forward(tape._h, -1.0, 0.9, 0.2, 0.0, 0.0, 1, 0.5, y.data_ptr(), 10, tape._ll.data_ptr())
    assert rc == 4                                        # BPF_ERR_UNSUPPORTED: ESS-mode tapes
    rc = lib.gpu_bpf_grad_forward(tape._h, -1.0, 0.9, 0.2, 0.0, 0.0, 1, 0.0, y.data_ptr(), 11, tape._ll.data_ptr())
    assert rc == 1                                        # more ticks than the tape holds
    rc = lib.gpu_bpf_grad_forward(tape._h, -1.0, 1.0, 0.2, 0.0, 0.0, 1, 0.0, y.data_ptr(), 10, tape._ll.data_ptr())
    assert rc == 1                                        # |rho| >= 1
    tape.close()
