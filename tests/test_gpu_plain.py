"""GPU parity tests of the plain filter, through the C ABI (libgpubpf.so), against
the CPU oracle (oracle/bpf_oracle.c) and the reference fixtures.

Tolerances
  PCG32 draws, ancestors           bit-exact
  normals vs exact inverse CDF     |dz| <= 1e-6 for |u-1/2| <= 0.425, <= 2e-6 in the tails
  per-tick log-lik increment       |d| <= 2e-4 absolute (FP32 particles vs FP64 oracle on
                                   replayed ancestors)
  total log-likelihood             <= 1e-4 relative
  filtered mean, ESS               |dh| <= 2e-4, ESS <= 1e-4 relative
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def series(T, seed, rho=RHO, sig=SIG, mu=MU):
    from gpubpf import dgp
    hs, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(hs), np.asarray(ys, dtype=np.float32)


def run_recorded(bpf, N, y, seed=42, thr=0.0, nu_obs=0.0, rho=RHO, sig=SIG, mu=MU, check_anc=None):
    """Tick-by-tick run that records every tick's ancestors; optionally checks each
    resampling tick's ancestors against check_anc(w, tile_exp, u23)."""
    f = bpf.GpuBpf(N, rho, sig, mu, 0.0, nu_obs, seed, ess_threshold=thr)
    f.record_ancestors(True)
    T = len(y)
    recs, flags = [], np.zeros(T, dtype=np.int32)
    anc = np.zeros((T, N), dtype=np.int32)
    for t in range(T):
        f.step(float(y[t]))
        recs.append(f.get_record())
        res, a = f.get_ancestors()
        flags[t] = int(res)
        if res:
            anc[t] = np.frombuffer(a, dtype=np.int32)
            if check_anc is not None:
                w, te, u23 = f.get_resample_inputs()
                check_anc(np.frombuffer(w, dtype=np.float32), np.frombuffer(te, dtype=np.int32), u23, anc[t])
    f.close()
    return recs, flags, anc


def rec_arrays(recs):
    return {
        "dll": np.array([r.dloglik for r in recs]),
        "ll_ref": np.array([r.loglik_ref for r in recs]),
        "total": np.array([r.loglik_total for r in recs]),
        "hmean": np.array([r.h_mean for r in recs], dtype=np.float64),
        "ess": np.array([r.ess for r in recs], dtype=np.float64),
        "res": np.array([r.resampled for r in recs]),
    }


# ---------------------------------------------------------------------------
# random numbers
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("seed", [42, 7, -3])
def test_device_pcg32_bit_exact(bpf, orc, seed):
    n = 5003
    for t in (0, 1, 2, 17, 1000, 4999):
        dev = bpf.debug_pcg32(seed, n, t)
        for i in list(range(0, 64)) + list(range(4090, 4110)) + [n - 1]:
            assert dev[i] == orc.pcg32_draw(seed, i, t), (seed, t, i)
    # every slot of one draw
    dev = bpf.debug_pcg32(seed, n, 5)
    assert dev == [orc.pcg32_draw(seed, i, 5) for i in range(n)]


def test_device_pcg32_reference_kat(bpf, golden):
    g = golden("rng_diag_seed42.json")
    dev = bpf.debug_pcg32(42, 8, 0)
    assert dev == [int(r["pcg_out"], 16) for r in g["rows"]]


def test_device_normals_accuracy(bpf, orc):
    L = orc.lib()
    n = 200_000
    outs = bpf.debug_pcg32(11, n, 3)
    z = np.asarray(bpf.debug_normals(11, n, 3), dtype=np.float64)
    assert np.all(np.isfinite(z))
    worst_c, worst_t = 0.0, 0.0
    for i in range(0, n, 7):
        u = L.orc_uniform(outs[i])
        e = abs(z[i] - L.orc_icdf_f64(u))
        if abs(u - 0.5) <= 0.425:
            worst_c = max(worst_c, e)
        else:
            worst_t = max(worst_t, e)
    assert worst_c <= 1e-6 and worst_t <= 2e-6, (worst_c, worst_t)
    # moments of tests/test_icdf_diag.cu:98 (N(0,1))
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01


# ---------------------------------------------------------------------------
# ancestors: bit-exact against the oracle on the same weights
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("N,thr,T", [(1, 0.0, 5), (2, 0.0, 8), (31, 0.5, 20), (4096, 0.0, 20), (4097, 0.5, 30),
                                     (100_003, 0.0, 6), ((1 << 20) + 3, 0.5, 6)])
def test_ancestors_bit_exact(bpf, orc, N, thr, T):
    _, y = series(T, 42)
    n_checked = []

    def check(w, te, u23, anc):
        ref = orc.resample_fixed(w, te, u23)
        np.testing.assert_array_equal(anc, ref)
        assert np.all(np.diff(anc) >= 0) and anc.min() >= 0 and anc.max() < N
        n_checked.append(1)

    run_recorded(bpf, N, y, seed=5, thr=thr, check_anc=check)
    assert len(n_checked) >= 1


@pytest.mark.parametrize("N", [8192, 12388, 40000])
def test_ancestors_adversarial_ties(bpf, orc, N):
    """A huge outlier observation concentrates the weight on few particles; the
    resampling must still be bit-exact and every output must land on a particle.
    With N > 8192 the heaviest tile owns more outputs than one pass-2 work window,
    so its outputs are split over several windows and single parents span them."""
    y = np.array([0.1, 0.2, 25.0, -0.3, 0.0, 40.0, 0.05], dtype=np.float32)
    split = []

    def check(w, te, u23, anc):
        np.testing.assert_array_equal(anc, orc.resample_fixed(w, te, u23))
        counts = np.bincount(anc // 4096, minlength=(N + 4095) // 4096)
        split.append(int(counts.max()))

    recs, flags, _ = run_recorded(bpf, N, y, seed=9, thr=0.0, check_anc=check)
    assert all(math.isfinite(r.dloglik) for r in recs)
    if N > 8192:
        assert max(split) > 8192          # the multi-window path ran


# ---------------------------------------------------------------------------
# log-likelihood against the FP64 oracle (ancestors replayed)
# ---------------------------------------------------------------------------
def compare_with_oracle(orc, N, y, seed, thr, recs, flags, anc, nu_obs=0.0, rho=RHO, sig=SIG, mu=MU):
    g = rec_arrays(recs)
    o = orc.filter_f64(N, rho, sig, mu, y, seed=seed, ess_threshold=thr, nu_obs=nu_obs,
                       anc_replay=anc, flags_replay=flags)
    np.testing.assert_array_equal(g["res"], flags)
    d = np.abs(g["dll"] - o["dll"])
    assert d.max() <= 2e-4, (d.max(), int(d.argmax()))
    tot_g, tot_o = g["dll"].sum(), o["dll"].sum()
    assert abs(tot_g - tot_o) / abs(tot_o) <= 1e-4, (tot_g, tot_o)
    assert abs(g["total"][-1] - tot_g) <= 1e-9 * abs(tot_g)
    assert np.max(np.abs(g["hmean"] - o["hmean"])) <= 2e-4
    assert np.max(np.abs(g["ess"] - o["ess"]) / o["ess"]) <= 1e-4
    assert np.max(np.abs(g["ll_ref"] - o["ll_ref"])) <= 2e-3
    return g, o


def test_config1_always_resample_vs_fp64_oracle(bpf, orc):
    """N=4096, T=1000, always resample, DGP seed 42, filter seed 42."""
    _, y = series(1000, 42)
    recs, flags, anc = run_recorded(bpf, 4096, y, seed=42, thr=0.0)
    assert flags.sum() == 1000
    g, o = compare_with_oracle(orc, 4096, y, 42, 0.0, recs, flags, anc)
    # always-resample: the reference's cumulative value equals the increment
    np.testing.assert_allclose(g["ll_ref"], g["dll"], rtol=0, atol=1e-12)


def test_ess_mode_vs_fp64_oracle(bpf, orc):
    """Config-2 semantics (ESS < 0.5 N, DGP seed 7) at N = 65536."""
    _, y = series(300, 7)
    recs, flags, anc = run_recorded(bpf, 65536, y, seed=7, thr=0.5)
    assert 0 < flags.sum() < 300
    g, o = compare_with_oracle(orc, 65536, y, 7, 0.5, recs, flags, anc)
    # the device decision matches ESS/N < 0.5 on the oracle's ESS except at a knife edge
    for t in range(300):
        r = o["ess"][t] / 65536
        if abs(r - 0.5) > 1e-5:
            assert flags[t] == int(r < 0.5), t


def test_student_t_observations(bpf, orc):
    _, y = series(200, 3)
    recs, flags, anc = run_recorded(bpf, 8192, y, seed=3, thr=0.5, nu_obs=5.0)
    compare_with_oracle(orc, 8192, y, 3, 0.5, recs, flags, anc, nu_obs=5.0)


def test_large_n_not_tile_multiple(bpf, orc):
    N = (1 << 22) + 5
    _, y = series(4, 42)

    def check(w, te, u23, anc):
        np.testing.assert_array_equal(anc, orc.resample_fixed(w, te, u23))

    recs, flags, anc = run_recorded(bpf, N, y, seed=1, thr=0.0, check_anc=check)
    compare_with_oracle(orc, N, y, 1, 0.0, recs, flags, anc)


# ---------------------------------------------------------------------------
# API semantics
# ---------------------------------------------------------------------------
def test_step_many_is_deterministic_and_matches_step(bpf):
    _, y = series(200, 42)
    a = bpf.GpuBpf(20_000, RHO, SIG, MU, seed=13, ess_threshold=0.5)
    b = bpf.GpuBpf(20_000, RHO, SIG, MU, seed=13, ess_threshold=0.5)
    ra = [a.step(float(v)) for v in y]
    rb = b.step_many(y.tolist(), records=True)
    for x, r in zip(ra, rb):
        assert x.h_mean == r.h_mean and x.log_lik == np.float32(r.dloglik)
    assert a.get_resample_count() == b.get_resample_count() == sum(r.resampled for r in rb)
    assert a.get_loglik_total() == b.get_loglik_total()
    ha = np.frombuffer(a.get_particles(), dtype=np.float32)
    hb = np.frombuffer(b.get_particles(), dtype=np.float32)
    np.testing.assert_array_equal(ha, hb)
    a.close(); b.close()


def test_loglik_reference_semantics(bpf):
    _, y = series(100, 42)
    f = bpf.GpuBpf(8192, RHO, SIG, MU, seed=2, ess_threshold=0.5)
    f.set_loglik_semantics(1)
    for v in y:
        r = f.step(float(v))
        rec = f.get_record()
        assert r.log_lik == np.float32(rec.loglik_ref)
    f.close()


def test_run_rmse_matches_oracle(bpf, orc):
    hs, y = series(1000, 42)
    rmse = bpf.run_rmse(y.astype(np.float64).tolist(), hs.tolist(), 4096, RHO, SIG, MU, seed=42)
    o = orc.filter_f64(4096, RHO, SIG, MU, y, seed=42, ess_threshold=0.5)
    rmse_o = math.sqrt(np.mean((o["hmean"][100:] - hs[100:]) ** 2))
    assert rmse < 0.8 and abs(rmse - rmse_o) < 0.03


def test_errors_are_reported(bpf):
    from gpubpf import _lib
    f = bpf.GpuBpf(4096, RHO, SIG, MU, seed=1)
    with pytest.raises(bpf.BpfError) as e:
        f.step(float("nan"))
    assert e.value.code == _lib.BPF_ERR_ARG
    f.state.silverman_shrink = float("nan")
    with pytest.raises(bpf.BpfError) as e:
        f.step(0.1)
    assert e.value.code == _lib.BPF_ERR_ARG
    f.state.silverman_shrink = 0.0
    f.step(0.1)
    f.set_rho(1.5)
    assert f.get_rho() == np.float32(0.999)
    f.close()


def test_parameters_change_between_ticks(bpf, orc):
    """set_mu between ticks takes effect on the next tick (graph and direct paths)."""
    _, y = series(130, 42)
    a = bpf.GpuBpf(4096, RHO, SIG, MU, seed=4, ess_threshold=0.0)
    b = bpf.GpuBpf(4096, RHO, SIG, MU, seed=4, ess_threshold=0.0)
    ra = a.step_many(y[:65].tolist(), records=True)
    rb = [b.step(float(v)) for v in y[:65]]
    a.set_mu(-0.5); b.set_mu(-0.5)
    ra += a.step_many(y[65:].tolist(), records=True)
    rb += [b.step(float(v)) for v in y[65:]]
    for x, r in zip(rb, ra):
        assert x.h_mean == r.h_mean
    a.close(); b.close()


def test_single_tick_graph_matches_direct_launches(bpf):
    """gpu_bpf_step (one captured tick graph, pass 1's observation updated per call) against
    gpu_bpf_step_async + get_record (direct launches), with mu, the ESS threshold and ancestor
    recording changed between ticks (each change re-captures the graph): identical records and
    ancestors."""
    _, y = series(90, 7)
    a = bpf.GpuBpf(5000, RHO, SIG, MU, seed=12, ess_threshold=0.5)
    b = bpf.GpuBpf(5000, RHO, SIG, MU, seed=12, ess_threshold=0.5)
    for t, v in enumerate(y):
        if t == 30:
            a.set_mu(-0.6); b.set_mu(-0.6)
        if t == 50:
            a.set_ess_threshold(0.0); b.set_ess_threshold(0.0)
        if t == 70:
            a.record_ancestors(True); b.record_ancestors(True)
        ra = a.step(float(v))
        rec_a = a.get_record()
        b.step_async(float(v))
        rec_b = b.get_record()
        assert (rec_a.dloglik, rec_a.h_mean, rec_a.ess, rec_a.resampled, rec_a.tick) == \
               (rec_b.dloglik, rec_b.h_mean, rec_b.ess, rec_b.resampled, rec_b.tick), t
        assert ra.h_mean == rec_a.h_mean
        if t >= 70:
            fa, aa = a.get_ancestors()
            fb, ab = b.get_ancestors()
            assert fa == fb and bytes(aa) == bytes(ab), t
    assert a.state.resample_count == b.state.resample_count and a.state.timestep == b.state.timestep == len(y)
    assert bytes(a.get_particles()) == bytes(b.get_particles())
    a.close(); b.close()


def test_independent_filters_do_not_interact(bpf):
    _, y = series(50, 42)
    solo = bpf.GpuBpf(10_000, RHO, SIG, MU, seed=21, ess_threshold=0.5)
    r_solo = [solo.step(float(v)).log_lik for v in y]
    solo.close()
    a = bpf.GpuBpf(10_000, RHO, SIG, MU, seed=21, ess_threshold=0.5)
    b = bpf.GpuBpf(30_000, 0.9, 0.3, 0.0, seed=22, ess_threshold=0.0)
    r_a = []
    for v in y:
        a.step_async(float(v)); b.step_async(float(-v))
        r_a.append(a.get_result().log_lik)
        b.get_result()
    assert r_a == r_solo
    a.close(); b.close()


# ---------------------------------------------------------------------------
# fused small-filter tick (N <= 65536): bit-identical to the three-kernel tick
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("N,thr,nu_obs,nu_state", [(1, 0.0, 0.0, 0.0), (31, 0.5, 0.0, 0.0), (4096, 0.0, 0.0, 0.0),
                                                   (4097, 0.5, 5.0, 0.0), (8192, 0.0, 0.0, 0.0),
                                                   (9000, 0.5, 0.0, 0.0), (12388, 0.5, 0.0, 5.0),
                                                   (16384, 0.3, 5.0, 5.0), (20000, 0.0, 0.0, 0.0),
                                                   (32768, 0.5, 5.0, 0.0), (40000, 0.0, 0.0, 5.0),
                                                   (65536, 0.5, 0.0, 0.0)])
def test_fused_small_matches_three_kernel_path(bpf, N, thr, nu_obs, nu_state):
    """Records, ancestors and particles of the fused one-launch tick equal the three-kernel
    tick's bit for bit: through step_many (a captured run of 64 ticks as one launch), the
    single-tick graph of gpu_bpf_step, and direct gpu_bpf_step_async launches."""
    _, y = series(150, 7)

    def run(fused, mode):
        f = bpf.GpuBpf(N, RHO, SIG, MU, nu_state, nu_obs, 17, ess_threshold=thr)
        f.set_fused_small(fused)
        f.record_ancestors(True)
        recs, ancs = [], []
        if mode == "many":
            recs = f.step_many(y[:128].tolist(), records=True)
            for v in y[128:]:
                f.step(float(v))
                recs.append(f.get_record())
                ancs.append(bytes(f.get_ancestors()[1]))
        else:
            for v in y:
                if mode == "step":
                    f.step(float(v))
                else:
                    f.step_async(float(v))
                recs.append(f.get_record())
                ancs.append(bytes(f.get_ancestors()[1]))
        parts = bytes(f.get_particles())
        w, te, u23 = f.get_resample_inputs()
        total = f.get_loglik_total()
        count = f.get_resample_count()
        f.close()
        key = [(r.dloglik, r.loglik_ref, r.loglik_total, r.h_mean, r.ess, r.resampled, r.tick) for r in recs]
        return key, ancs, parts, bytes(w), bytes(te), u23, total, count

    for mode in ("many", "step", "async"):
        a = run(True, mode)
        b = run(False, mode)
        assert a[0] == b[0], mode
        assert a[1] == b[1] and a[2] == b[2] and a[3:] == b[3:], mode


@pytest.mark.parametrize("N,thr", [(4096, 0.0), (12000, 0.5), (16384, 0.0), (30000, 0.5), (65536, 0.0)])
def test_fused_small_long_device_run(bpf, N, thr):
    """A whole device-resident run of 2500 ticks as one fused launch (one CTA, or a cluster of
    3, 4, 8 or 16, padding CTAs included; the observations are restaged in shared memory every
    1024 ticks) equals the three-kernel run."""
    import torch
    T = 2500
    _, y = series(T, 42)
    yd = torch.tensor(y, device="cuda")
    out = []
    for fused in (True, False):
        f = bpf.GpuBpf(N, RHO, SIG, MU, seed=42, ess_threshold=thr)
        f.set_fused_small(fused)
        rec = torch.zeros(T * 40, dtype=torch.uint8, device="cuda")
        f.step_many_device(yd.data_ptr(), T, rec.data_ptr())
        torch.cuda.synchronize()
        w, te, u23 = f.get_resample_inputs()
        out.append((rec.cpu().numpy().tobytes(), bytes(f.get_particles()), bytes(w), bytes(te), u23))
        f.close()
    assert out[0] == out[1]


@pytest.mark.parametrize("N,thr", [(65537, 0.0), (100000, 0.5), (300000, 0.5), (1 << 20, 0.0)])
def test_tail_plan_matches_plan_kernel(bpf, N, thr):
    """Filters of at most 256 tiles run the plan in pass 1's last CTA; with per-kernel profiling
    on, the same ticks run the separate plan kernel. Records, ancestors and particles agree bit
    for bit, tick by tick and over a captured run."""
    _, y = series(120, 11)

    def run(profile):
        f = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 23, ess_threshold=thr)
        f.record_ancestors(True)
        if profile:
            f.profile(True)
        recs, ancs = [], []
        for v in y[:40]:
            f.step(float(v))
            recs.append(f.get_record())
            ancs.append(bytes(f.get_ancestors()[1]))
        recs += f.step_many(y[40:].tolist(), records=True)
        parts = bytes(f.get_particles())
        f.close()
        key = [(r.dloglik, r.loglik_ref, r.loglik_total, r.h_mean, r.ess, r.resampled, r.tick) for r in recs]
        return key, ancs, parts

    a, b = run(False), run(True)
    assert sum(r[5] for r in a[0]) > 0
    assert a[0] == b[0]
    assert a[1] == b[1] and a[2] == b[2]
