"""GPU parity at the headline sizes of the scaling configuration (SV model mu=-1, phi=0.97,
sigma_eta=0.15, observations of the matched DGP with seed 7, resampling when ESS < 0.5 N).

The device filter runs tick by tick through the C ABI; the FP64 oracle (oracle.F64Filter) follows
it in lock step, replaying each tick's resampling decision and, on resampling ticks, the device's
ancestors, so both work on the same particle cloud and the log-likelihoods can be compared at any
run length. On every resampling tick the device's ancestors are also recomputed by the oracle's
mirror of the fixed-point systematic resampling from the device's own weights, and must agree
bit for bit. At N = 2^24 the global fixed-point frame has 38 fraction bits and at 51 200 000 it
has 36 (Fg = min(50, 62 - ceil(log2 N))): the sizes where an FP32 CDF loses whole particles.

Tolerances
  ancestors                      bit-exact (against the oracle's fixed-point mirror)
  per-tick log-lik increment     |d| <= 2e-4 absolute
  total log-likelihood           <= 1e-4 relative
  filtered mean                  |dh| <= 2e-4
  ESS                            <= 1e-4 relative
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def series(T, seed):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(ys, dtype=np.float32)


def lockstep(bpf, orc, N, y, seed, thr, always_after=None, check_ancestors=True, min_resamples=0):
    """Run the device filter and the FP64 oracle side by side over y. From tick `always_after` on
    the device resamples every tick (threshold 0). Returns per-tick arrays and counts."""
    f = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, seed, ess_threshold=thr)
    f.record_ancestors(True)
    o = orc.F64Filter(N, RHO, SIG, MU, seed=seed, ess_threshold=thr)
    T = len(y)
    g_dll, o_dll = np.zeros(T), np.zeros(T)
    g_h, o_h = np.zeros(T), np.zeros(T)
    g_e, o_e = np.zeros(T), np.zeros(T)
    flags = np.zeros(T, dtype=np.int32)
    n_anc_checked = 0
    last_total = 0.0
    try:
        for t in range(T):
            if always_after is not None and t == always_after:
                f.set_ess_threshold(0.0)
            f.step(float(y[t]))
            r = f.get_record()
            flags[t] = r.resampled
            anc = None
            if r.resampled:
                ok, a = f.get_ancestors()
                assert ok
                anc = np.frombuffer(a, dtype=np.int32)
                if check_ancestors:
                    w, te, u23 = f.get_resample_inputs()
                    ref = orc.resample_fixed(np.frombuffer(w, dtype=np.float32), np.frombuffer(te, dtype=np.int32),
                                             u23)
                    if not np.array_equal(anc, ref):
                        bad = np.flatnonzero(anc != ref)
                        raise AssertionError(f"tick {t}: {bad.size} ancestors differ, first at {bad[0]}: "
                                             f"{anc[bad[0]]} vs {ref[bad[0]]}")
                    n_anc_checked += 1
            q = o.tick(y[t], anc=anc, flag=int(r.resampled))
            g_dll[t], o_dll[t] = r.dloglik, q["dll"]
            g_h[t], o_h[t] = r.h_mean, q["hmean"]
            g_e[t], o_e[t] = r.ess, q["ess"]
            last_total = r.loglik_total
    finally:
        f.close()
        o.close()
    assert n_anc_checked >= min_resamples, n_anc_checked
    return {"g_dll": g_dll, "o_dll": o_dll, "g_h": g_h, "o_h": o_h, "g_e": g_e, "o_e": o_e, "flags": flags,
            "n_anc": n_anc_checked, "total": last_total}


def assert_parity(r):
    d = np.abs(r["g_dll"] - r["o_dll"])
    assert d.max() <= 2e-4, (d.max(), int(d.argmax()))
    tg, to = r["g_dll"].sum(), r["o_dll"].sum()
    assert abs(tg - to) / abs(to) <= 1e-4, (tg, to)
    assert abs(r["total"] - tg) <= 1e-9 * abs(tg)
    assert np.max(np.abs(r["g_h"] - r["o_h"])) <= 2e-4
    assert np.max(np.abs(r["g_e"] - r["o_e"]) / r["o_e"]) <= 1e-4
    return abs(tg - to) / abs(to)


def test_headline_n_2p24(bpf, orc):
    """N = 2^24: 24 ticks of the ESS rule, then 3 always-resampling ticks; every resampling tick's
    ancestors bit-exact, increments and the total against the FP64 oracle."""
    y = series(27, 7)
    r = lockstep(bpf, orc, 1 << 24, y, seed=7, thr=0.5, always_after=24, min_resamples=3)
    assert r["flags"][:24].sum() < 24          # the ESS rule skipped some ticks (carried weights)
    rel = assert_parity(r)
    print(f"N=2^24: {r['n_anc']} resampling ticks bit-exact, total loglik rel err {rel:.2e}")


def test_headline_n_51p2m(bpf, orc):
    """N = 51 200 000 (the sweep's largest point, 36 fraction bits in the global frame)."""
    y = series(23, 7)
    r = lockstep(bpf, orc, 51_200_000, y, seed=7, thr=0.5, always_after=20, min_resamples=3)
    rel = assert_parity(r)
    print(f"N=51.2M: {r['n_anc']} resampling ticks bit-exact, total loglik rel err {rel:.2e}")


def test_config2_full_series_n_2p20(bpf, orc):
    """The scaling configuration over its whole T = 5000 series at N = 2^20 (ESS < 0.5 N):
    every resampling tick's ancestors bit-exact and the FP64 oracle followed for all 5000 ticks."""
    y = series(5000, 7)
    r = lockstep(bpf, orc, 1 << 20, y, seed=7, thr=0.5, min_resamples=50)
    assert 0 < r["flags"].sum() < 5000
    rel = assert_parity(r)
    print(f"N=2^20, T=5000: {r['n_anc']} resampling ticks bit-exact, total loglik rel err {rel:.2e}")
