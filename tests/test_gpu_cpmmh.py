"""GPU tests of correlated-noise runs (gpu_bpf_batch_run_correlated) and the SMC^2 driver's
correlated-noise PMMH moves (gpu_bpf_smc2_set_cpmmh_rho; the reference's CPMMH rejuvenation,
smc2/smc2_rbpf_batch.cu:651-935, and smc2_cuda_set_cpmmh_rho :1238-1240).

  fresh run (no input noise; Gaussian    recorded normals equal the filters' PCG32 draws bit for bit
  and Student-t observations)
                                        (slot kBatchMaxN = 16384 for the resampling normal); the
                                        FP64 oracle driven by the recorded noise, the GPU's
                                        resampling decisions and slot ancestors: per-tick dll <= 2e-4
                                        absolute, total dll <= 1e-4 relative; the ancestors visit the
                                        sorted particles in order; in lock step the oracle's own
                                        sorted systematic resampling picks the same ancestor for
                                        >= 99% of the slots, the others a sorted neighbour (FP32
                                        weights and the fixed-point CDF against FP64)
  rho = 1 with other seeds              the noise is replayed: output noise, log-likelihoods,
                                        per-tick increments identical bit for bit
  0 < rho < 1                           output noise = fmaf(rho, input, sqrt(1-rho^2) * fresh) within
                                        one FP32 ulp; log-likelihood differences between the run
                                        and its correlated re-run shrink with rho (the CPMMH effect)
  SMC^2, rho = 1, tiny proposal steps   after every update each theta-particle's noise is one held
                                        before it (bit for bit); proposals score within 0.5 nats
                                        (median 0.05) of the current inner log-likelihood
  SMC^2, rho = 0.99 vs fresh filters    64 state particles (estimator noise dominates): acceptance
                                        at least 1.2x that of fresh inner filters at the same
                                        proposal scale, posterior around the generating theta
  argument checks                       rho outside [0, 1], switching after the first update, more
                                        than 4096 particles, Student-t state noise
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def _series(T, theta=(MU, RHO, SIG), seed=42):
    from gpubpf import dgp
    mu, rho, sig = theta
    _, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def _filters(ns, seed0=100, nu_obs=None):
    rng = np.random.default_rng(4)
    out = []
    for j, n in enumerate(ns):
        out.append({"mu": float(rng.normal(-1.0, 0.3)), "rho": float(rng.uniform(0.9, 0.99)),
                    "sigma_z": float(rng.uniform(0.1, 0.3)), "n_particles": int(n), "seed": seed0 + j,
                    "nu_obs": float(nu_obs[j]) if nu_obs is not None else 0.0})
    return out


def _stride(n):
    return ((n + 3) & ~3) + 4


def _run(bpf, b, y_dev, T, nin, nout, rho, B, anc=False):
    import torch
    ll = torch.zeros(B, dtype=torch.float64, device="cuda")
    dll = torch.zeros(B * T, dtype=torch.float64, device="cuda")
    a = torch.full((B * T * 16384,), -1, dtype=torch.int32, device="cuda") if anc else None
    b.run_correlated(y_dev.data_ptr(), T, nin.data_ptr() if nin is not None else 0, nout.data_ptr(), rho,
                     ll.data_ptr(), dll.data_ptr(), a.data_ptr() if anc else 0)
    torch.cuda.synchronize()
    out = {"ll": ll.cpu().numpy(), "dll": dll.cpu().numpy().reshape(B, T)}
    if anc:
        out["anc"] = a.cpu().numpy().reshape(B, T, 16384)
    return out


def _area(b, nz, f, T, n):
    off = b.noise_offset(f, T)
    return nz[off:off + T * _stride(n)].reshape(T, _stride(n))


def test_fresh_run_records_pcg_noise_and_matches_oracle(bpf, orc):
    import torch
    lib = bpf.load()
    ns = [512, 1000, 4096, 37, 800]
    T = 60
    fl = _filters(ns, nu_obs=[0.0, 0.0, 0.0, 0.0, 5.0])        # the last one: Student-t observations
    y = _series(T)
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    nfl = b.noise_offset(len(ns), T)
    nz = torch.full((nfl,), float("nan"), dtype=torch.float32, device="cuda")
    y_dev = torch.tensor(y, device="cuda")
    r = _run(bpf, b, y_dev, T, None, nz, 0.0, len(ns), anc=True)
    nzh = nz.cpu().numpy()
    areas = [_area(b, nzh, f, T, n) for f, n in enumerate(ns)]
    b.close()
    import ctypes as C
    agree = total = 0
    for f, (fd, n) in enumerate(zip(fl, ns)):
        z = areas[f]
        for t in (0, 1, T // 2, T - 1):
            ref = (C.c_float * 16385)()
            assert lib.gpu_bpf_debug_normals(fd["seed"], 16385, t, ref) == 0
            ref = np.frombuffer(ref, dtype=np.float32)
            np.testing.assert_array_equal(z[t, :n], ref[:n])
            assert z[t, _stride(n) - 4] == ref[16384]
        anc = r["anc"][f, :, :n]
        flags = (anc[:, 0] >= 0).astype(np.int32)          # resampling ticks wrote their ancestors
        assert flags.sum() > 0
        o = orc.filter_noise_f64(n, fd["rho"], fd["sigma_z"], fd["mu"], y, z, ess_threshold=0.5,
                                 nu_obs=fd["nu_obs"], anc_replay=np.maximum(anc, 0), flags_replay=flags)
        np.testing.assert_array_equal(o["resampled"], flags)
        np.testing.assert_allclose(r["dll"][f], o["dll"], atol=2e-4, rtol=0)
        assert abs(r["dll"][f].sum() - o["dll"].sum()) <= 1e-4 * abs(o["dll"].sum())
        assert abs(r["ll"][f] - r["dll"][f].sum()) <= 1e-9 * abs(r["ll"][f])
        # the ancestors visit the particles in ascending order (oracle particles, FP64)
        sstat = math.sqrt(np.float32(fd["sigma_z"]) ** 2 / max(1 - np.float32(fd["rho"]) ** 2, 1e-6))
        h = np.float32(fd["mu"]) + sstat * z[0, :n].astype(np.float64)
        for t in range(T):
            if t > 0:
                h = fd["mu"] + fd["rho"] * (h - fd["mu"]) + fd["sigma_z"] * z[t, :n].astype(np.float64)
            if flags[t]:
                a, own = anc[t], o["anc"][t]
                assert a.min() >= 0 and a.max() < n
                assert np.all(np.diff(h[a]) >= -1e-5), (f, t)
                rank = np.empty(n, dtype=np.int64)
                rank[np.lexsort((np.arange(n), h))] = np.arange(n)
                assert np.all(np.abs(rank[a] - rank[own]) <= 2), (f, t)
                total += n
                agree += int(np.sum(a == own))
                h = h[a]
    assert agree >= 0.99 * total, (agree, total)


def test_rho_one_replays_the_noise_exactly(bpf):
    import torch
    ns = [512, 2000, 4096]
    T = 80
    fl = _filters(ns)
    y_dev = torch.tensor(_series(T, seed=3), device="cuda")
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    nfl = b.noise_offset(len(ns), T)
    na = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    nb = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    ra = _run(bpf, b, y_dev, T, None, na, 0.0, len(ns))
    b.set_filters([dict(f, seed=f["seed"] + 7777) for f in fl])
    rb = _run(bpf, b, y_dev, T, na, nb, 1.0, len(ns))
    b.close()
    assert torch.equal(na, nb)
    np.testing.assert_array_equal(ra["ll"], rb["ll"])
    np.testing.assert_array_equal(ra["dll"], rb["dll"])


def test_partial_correlation_mixes_the_noise(bpf):
    import torch
    import ctypes as C
    lib = bpf.load()
    ns = [700, 1024]
    T = 50
    fl = _filters(ns)
    y_dev = torch.tensor(_series(T, seed=9), device="cuda")
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    nfl = b.noise_offset(len(ns), T)
    na = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    nb = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    _run(bpf, b, y_dev, T, None, na, 0.0, len(ns))
    fl2 = [dict(f, seed=f["seed"] + 99) for f in fl]
    b.set_filters(fl2)
    rho = 0.9
    _run(bpf, b, y_dev, T, na, nb, rho, len(ns))
    b.close()
    ah, bh = na.cpu().numpy(), nb.cpu().numpy()
    cr = np.float32(rho)
    cs = np.sqrt(np.float32(1.0) - cr * cr)           # FP32 throughout, as the host computes it
    off = 0
    for f, n in enumerate(ns):
        s = _stride(n)
        za = ah[off:off + T * s].reshape(T, s)
        zb = bh[off:off + T * s].reshape(T, s)
        off += T * s
        for t in (0, 1, T - 1):
            ref = (C.c_float * 16385)()
            assert lib.gpu_bpf_debug_normals(fl2[f]["seed"], 16385, t, ref) == 0
            fresh = np.frombuffer(ref, dtype=np.float32)
            fr = np.concatenate([fresh[:n], fresh[16384:16385]])
            zin = np.concatenate([za[t, :n], za[t, s - 4:s - 3]])
            got = np.concatenate([zb[t, :n], zb[t, s - 4:s - 3]])
            p = (cs * fr).astype(np.float32)
            want = (np.float64(cr) * zin.astype(np.float64) + p.astype(np.float64)).astype(np.float32)
            ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
            assert ulp.max() <= 1, (f, t, ulp.max())


def test_loglik_correlation_grows_with_rho(bpf):
    # the CPMMH effect: re-running with noise correlated to the current run's moves the
    # log-likelihood estimate far less than an independent run does
    import torch
    B, N, T = 64, 512, 300
    fl = [{"mu": -1.0, "rho": 0.97, "sigma_z": 0.15, "n_particles": N, "seed": 10 + j} for j in range(B)]
    y_dev = torch.tensor(_series(T, seed=21), device="cuda")
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.5)
    nfl = b.noise_offset(B, T)
    na = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    nb = torch.zeros(nfl, dtype=torch.float32, device="cuda")
    ra = _run(bpf, b, y_dev, T, None, na, 0.0, B)
    b.set_filters([dict(f, seed=f["seed"] + 1000) for f in fl])
    sd = {}
    for rho in (0.0, 0.9, 0.99):
        rb = _run(bpf, b, y_dev, T, na if rho > 0 else None, nb, rho, B)
        sd[rho] = float(np.std(rb["ll"] - ra["ll"]))
    b.close()
    print("sd of loglik differences by rho:", sd)
    assert sd[0.99] < sd[0.9] < sd[0.0]
    assert sd[0.99] < 0.3 * sd[0.0]


def test_smc2_cpmmh_rho_one_keeps_and_moves_the_noise(bpf):
    # rho = 1: proposals reuse the current noise exactly, so every theta-particle's noise after an
    # update is the noise some theta-particle held before it (outer resampling copies areas,
    # accepted moves flip to an identical copy), and with near-zero proposal steps (the
    # covariance jitter alone, ~1e-5) a proposal scores almost exactly the current estimate
    M, N, T = 32, 256, 80
    y = _series(T, theta=(-1.0, 0.95, 0.25), seed=5)
    s = bpf.Smc2(M, N, T, seed=11)
    s.set_moves(1, 0.5, 1e-20)
    s.set_cpmmh_rho(1.0)
    moves = 0
    last = 0
    for t, v in enumerate(y):
        before = set()
        if t > 0:
            for j in range(M):
                zz, rr = s.noise(j, t, N)
                before.add(zz.tobytes() + rr.tobytes())
        s.update(float(v))
        if t > 0:
            for j in range(M):
                zz, rr = s.noise(j, t, N)
                assert zz.tobytes() + rr.tobytes() in before, (t, j)
        st = s.stats()
        if st["rejuvenations"] > last:
            last = st["rejuvenations"]
            lm = s.last_move()
            d = np.abs(lm["loglik_prop"] - lm["loglik_cur"])
            assert np.median(d) < 0.05 and d.max() < 0.5, (t, d)
            moves += 1
    s.close()
    assert moves >= 2


def test_smc2_cpmmh_raises_acceptance(bpf):
    # 64 state particles over 400 ticks: independent estimates of the log-likelihood differ by
    # about 1.9 nats (sd), correlated ones (rho 0.99, sorted resampling) by about 0.6 (FP64 oracle
    # on the same noise model), so estimator noise, not the proposal, limits PMMH's acceptance
    truth = (-1.0, 0.95, 0.25)
    T = 400
    y = _series(T, truth, seed=11)
    res = {}
    for rho in (0.0, 0.99):
        s = bpf.Smc2(256, 64, T, seed=7)
        s.set_moves(2, 0.5, 0.5)
        s.set_cpmmh_rho(rho)
        for v in y:
            s.update(float(v))
        mean, sd = s.theta()
        st = s.stats()
        s.close()
        res[rho] = (st["accepted"] / max(1, st["proposed"]), mean, sd, st)
    print("acceptance: PMMH %.3f, CPMMH(0.99) %.3f" % (res[0.0][0], res[0.99][0]))
    assert res[0.99][0] > 1.2 * res[0.0][0], res
    _, mean, sd, st = res[0.99]
    assert st["rejuvenations"] >= 3
    assert abs(mean[0] - truth[0]) < 3 * sd[0] + 0.1, (mean, sd)
    assert abs(mean[2] - truth[2]) < 3 * sd[2] + 0.05, (mean, sd)
    assert 0.85 < mean[1] < 0.995


def test_cpmmh_argument_checks(bpf):
    import torch
    from gpubpf import BpfError
    s = bpf.Smc2(8, 256, 10, seed=1)
    with pytest.raises(BpfError):
        s.set_cpmmh_rho(1.5)
    with pytest.raises(BpfError):
        s.set_cpmmh_rho(-0.1)
    s.set_cpmmh_rho(0.5)
    s.set_cpmmh_rho(0.0)
    s.update(0.1)
    with pytest.raises(BpfError):
        s.set_cpmmh_rho(0.9)                     # switching on after the first update
    s.close()
    big = bpf.Smc2(4, 5000, 10, seed=1)
    with pytest.raises(BpfError):
        big.set_cpmmh_rho(0.9)                   # more than one 4096-particle tile
    big.close()
    y_dev = torch.zeros(4, dtype=torch.float32, device="cuda")
    nz = torch.zeros(1 << 16, dtype=torch.float32, device="cuda")
    ll = torch.zeros(1, dtype=torch.float64, device="cuda")
    b = bpf.GpuBpfBatch([{"mu": -1.0, "rho": 0.9, "sigma_z": 0.2, "n_particles": 100, "seed": 1, "nu_state": 5.0}])
    with pytest.raises(BpfError):
        b.run_correlated(y_dev.data_ptr(), 4, 0, nz.data_ptr(), 0.0, ll.data_ptr())
    b.close()
    b = bpf.GpuBpfBatch([{"mu": -1.0, "rho": 0.9, "sigma_z": 0.2, "n_particles": 100, "seed": 1}])
    with pytest.raises(BpfError):
        b.run_correlated(y_dev.data_ptr(), 4, nz.data_ptr(), nz.data_ptr(), 0.5, ll.data_ptr())   # in == out
    b.close()
