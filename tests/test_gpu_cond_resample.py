"""The reference's conditional-resampling study (tests/test_cond_resample.cu) with assertions: ESS
thresholds {always, 0.3, 0.5, 0.7, 0.9} on its four scenarios, this build against the reference's
own GPU filter (the PTX edition, whose Silverman jitter is off, as in this build) on the same series.

  scenarios (:124-200)     N = 300000, T = 3000, rho 0.98, sigma_z 0.15, mu -4.5, filter seed 42:
                           oracle parameters; filter sigma_z 0.08 (misspecified); a regime change
                           (sigma_z 0.15 -> 0.40 at t = 1500); high volatility (sigma_z 0.40)
  series                   gpubpf.dgp.cond_resample_series: the suite's host PCG32 + Box-Muller
                           generator restated in numpy FP32 (seed 42, :25-57); the same law, not
                           pinned bit for bit to the C build
  checks                   per scenario and threshold: resampling counts within 2% (+3) of the
                           reference's, RMSE of the filtered mean after 100 ticks within 0.01;
                           this build's count falls as the threshold falls
"""
from __future__ import annotations


import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T, N, SKIP = 3000, 300000, 100
RHO, SZ, MU = 0.98, 0.15, -4.5


def _series(sigma_of_t):
    from gpubpf import dgp
    h, y = dgp.cond_resample_series(sigma_of_t, T, RHO, MU, 42)
    return y, h


def _rmse(hm, h):
    e = np.asarray(hm[SKIP:], dtype=np.float64) - h[SKIP:]
    return float(np.sqrt(np.mean(e * e)))


def test_conditional_resampling_matches_reference(bpf):
    from oracle import refgpu
    if not refgpu.available():
        pytest.skip("oracle/_ref not built")
    y1, h1 = _series(lambda t: SZ)
    y3, h3 = _series(lambda t: SZ if t < 1500 else 0.40)
    y4, h4 = _series(lambda t: 0.40)
    scenarios = [("oracle params", y1, h1, SZ), ("wrong sigma_z 0.08", y1, h1, 0.08),
                 ("regime 0.15 -> 0.40", y3, h3, SZ), ("high vol 0.40", y4, h4, 0.40)]
    rows = []
    for name, y, h, sz in scenarios:
        counts = []
        for thr in (0.0, 0.3, 0.5, 0.7, 0.9):
            f = bpf.GpuBpf(N, RHO, sz, MU, seed=42, ess_threshold=thr)
            out = f.step_many(y.tolist())
            ours_n = f.state.resample_count
            f.close()
            ours_rmse = _rmse([r.h_mean for r in out], h)
            g = refgpu.RefGpuFilter(N, RHO, sz, MU, seed=42, ess_threshold=thr)
            hm, _ = g.run(y)
            ref_n = g.resample_count
            g.close()
            ref_rmse = _rmse(hm, h)
            rows.append((name, thr, ours_n, ref_n, ours_rmse, ref_rmse))
            counts.append(ours_n)
        assert counts[0] == T
        assert counts[1] <= counts[2] <= counts[3] <= counts[4] <= T, (name, counts)
    print("\n  scenario              thr   resamples ours / ref   RMSE ours / ref")
    for name, thr, on, rn, orm, rrm in rows:
        print(f"  {name:20s}  {thr:3.1f}   {on:5d} / {rn:5d}          {orm:.4f} / {rrm:.4f}")
    for name, thr, on, rn, orm, rrm in rows:
        assert abs(on - rn) <= 3 + 0.02 * rn, (name, thr, on, rn)
        assert abs(orm - rrm) <= 0.01, (name, thr, orm, rrm)
