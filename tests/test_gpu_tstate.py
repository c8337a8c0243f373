"""GPU tests of Student-t state noise (nu_state > 0) through the C ABI.

The reference draws eps = z * sqrt(nu_state / chi2), chi2 a sum of round(nu_state)
squared normals from a separate cuRAND stream (gpu_bpf/gpu_bpf_ptx_full.cu:392-400,
574-583; ptx_assembly/bpf_kernels_full.ptx:394-404). This build draws the same law
from counter-based PCG32 streams (oracle/bpf_oracle.c orc_tstate_scale restates it in
FP64), so the checks are:
  noise vs the FP64 oracle's draws       |d eps| <= 2e-5 * max(1, |eps|)
  noise moments (reference test          mean 0, std sqrt(5/3) = 1.291
  tests/test_icdf_diag.cu:251-253)
  total loglik vs FP64 oracle (replayed  <= 1e-4 relative; per tick <= 2e-4 absolute
  ancestors and decisions)
  batched vs plain                       ancestors and particles bit-exact
  adjoint vs FP64 oracle adjoint         <= 1e-4 relative to the largest component
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(T, seed=42):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, 0.97, 0.15, -1.0, seed)
    return np.asarray(ys, dtype=np.float32)


def test_tstate_noise_matches_oracle_draws(bpf, orc):
    # rho = 0, sigma = 1, mu = 0, no resampling: the particles after tick 1 are the noise itself
    N, seed = 100000, 42
    f = bpf.GpuBpf(N, 0.0, 1.0, 0.0, 5.0, 0.0, seed, ess_threshold=1e-9)
    f.step(0.3)
    f.step(-0.2)
    assert f.get_record().resampled == 0
    eps = np.frombuffer(f.get_particles(), dtype=np.float32).astype(np.float64)
    f.close()
    assert np.all(np.isfinite(eps))
    assert abs(eps.mean()) < 0.02
    assert abs(eps.std() - math.sqrt(5.0 / 3.0)) < 0.03
    L = orc.lib()
    n = 5000
    ref = np.array([L.orc_icdf_f64(L.orc_uniform(L.orc_pcg32_draw_jump(seed, i, 1))) *
                    L.orc_tstate_scale(seed, i, 1, 5, 5.0) for i in range(n)])
    err = np.abs(eps[:n] - ref) / np.maximum(1.0, np.abs(ref))
    assert err.max() <= 2e-5, err.max()


@pytest.mark.parametrize("thr", [0.0, 0.5])
def test_tstate_filter_matches_fp64_oracle(bpf, orc, thr):
    N, T, seed = 4096, 80, 42
    y = _series(T)
    f = bpf.GpuBpf(N, 0.97, 0.15, -1.0, 5.0, 5.0, seed, ess_threshold=thr)
    f.record_ancestors(True)
    dll = np.zeros(T)
    anc = np.zeros((T, N), dtype=np.int32)
    flags = np.zeros(T, dtype=np.int32)
    for t in range(T):
        f.step(float(y[t]))
        dll[t] = f.get_record().dloglik
        res, a = f.get_ancestors()
        flags[t] = res
        if res:
            anc[t] = np.frombuffer(a, dtype=np.int32)
    f.close()
    o = orc.filter_f64(N, 0.97, 0.15, -1.0, y, seed=seed, ess_threshold=thr, nu_obs=5.0, nu_state=5.0,
                       anc_replay=anc, flags_replay=flags)
    assert np.max(np.abs(dll - o["dll"])) <= 2e-4
    assert abs(dll.sum() - o["dll"].sum()) <= 1e-4 * abs(o["dll"].sum())


def test_tstate_batch_matches_plain(bpf):
    import torch
    fl = [{"mu": -1.0, "rho": 0.97, "sigma_z": 0.15, "n_particles": 3000, "seed": 3, "nu_state": 5.0},
          {"mu": -0.6, "rho": 0.9, "sigma_z": 0.3, "n_particles": 9000, "seed": 4, "nu_state": 3.0, "nu_obs": 5.0},
          {"mu": -1.2, "rho": 0.95, "sigma_z": 0.2, "n_particles": 700, "seed": 5, "nu_state": 0.0}]
    y = _series(30)
    B, T, MAXN = len(fl), len(y), 16384
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.0)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(B, dtype=torch.float64, device="cuda")
    anc = torch.full((B * T * MAXN,), -1, dtype=torch.int32, device="cuda")
    parts = torch.zeros(B * MAXN, dtype=torch.float32, device="cuda")
    b.run_debug(y_d.data_ptr(), T, ll.data_ptr(), 0, anc.data_ptr(), parts.data_ptr())
    torch.cuda.synchronize()
    b.close()
    anc = anc.cpu().numpy().reshape(B, T, MAXN)
    parts = parts.cpu().numpy().reshape(B, MAXN)
    for i, f in enumerate(fl):
        n = f["n_particles"]
        p = bpf.GpuBpf(n, f["rho"], f["sigma_z"], f["mu"], f["nu_state"], f.get("nu_obs", 0.0), f["seed"],
                       ess_threshold=0.0)
        p.record_ancestors(True)
        for t in range(T):
            p.step(float(y[t]))
            _, a = p.get_ancestors()
            np.testing.assert_array_equal(anc[i, t, :n], np.frombuffer(a, dtype=np.int32))
        np.testing.assert_array_equal(parts[i, :n], np.frombuffer(p.get_particles(), dtype=np.float32))
        p.close()


def test_tstate_adjoint_matches_fp64_oracle(bpf, orc):
    import torch
    N, T, seed, theta = 4096, 120, 42, (-0.8, 0.95, 0.25)
    y = _series(T)
    tape = bpf.GradTape(N, T, checkpoint_every=16)
    ll = tape.forward(theta, torch.tensor(y, device="cuda"), seed=seed, nu_obs=5.0, nu_state=5.0).item()
    g = tape.backward().cpu().numpy()
    rep = tape.replay(theta).cpu().numpy()
    anc = np.stack([tape.ancestors(t) for t in range(T)])
    tape.close()
    oll, og, _ = orc.grad_f64(N, *theta, y, anc, seed=seed, nu_obs=5.0, nu_state=5.0, mode=1)
    assert abs(ll - oll) <= 1e-4 * abs(oll)
    assert np.max(np.abs(g - og)) <= 1e-4 * np.max(np.abs(og)), (g, og)
    assert np.max(np.abs(g - rep[1:])) <= 1e-4 * np.max(np.abs(rep[1:]))


def test_tstate_batch_gradient_matches_plain_tape(bpf):
    import torch
    fl = [{"mu": -0.8, "rho": 0.95, "sigma_z": 0.25, "n_particles": 5000, "seed": 6, "nu_state": 5.0},
          {"mu": -1.1, "rho": 0.9, "sigma_z": 0.2, "n_particles": 2000, "seed": 7, "nu_state": 8.0}]
    y = _series(40)
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.0)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(2, dtype=torch.float64, device="cuda")
    gd = torch.zeros(6, dtype=torch.float64, device="cuda")
    b.grad_run(y_d.data_ptr(), len(y), ll.data_ptr(), gd.data_ptr())
    torch.cuda.synchronize()
    b.close()
    gd = gd.cpu().numpy().reshape(2, 3)
    for i, f in enumerate(fl):
        tape = bpf.GradTape(f["n_particles"], len(y), checkpoint_every=8)
        tape.forward((f["mu"], f["rho"], f["sigma_z"]), y_d, seed=f["seed"], nu_state=f["nu_state"])
        pg = tape.backward().cpu().numpy()
        tape.close()
        assert np.max(np.abs(gd[i] - pg)) <= 1e-4 * np.max(np.abs(pg)), (i, gd[i], pg)


def test_tstate_rejects_below_one_half(bpf):
    from gpubpf._lib import BpfError
    with pytest.raises(BpfError):
        bpf.GpuBpf(100, 0.9, 0.2, -1.0, 0.3, 0.0, 1)
