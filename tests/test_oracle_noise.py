"""The noise-driven FP64 oracle (orc_filter_noise_f64, the checker of correlated-noise runs)
against an independent numpy restatement of the same filter.

  noise layout        z[t, :N] the particles' normals (tick 0: h_0 = mu + s_stat z), z[t, stride-4]
                      the normal v_t of the tick's resampling offset Phi(v_t) on the 23-bit grid
                      (the reference stores the same per-tick noise for its CPMMH replay,
                      smc2/smc2_rbpf_batch.cu:741-860)
  resampling          particles sorted by value (ties by slot) before every systematic resampling
  checks              per-tick dll / hmean / ess <= 1e-12 relative, resampling decisions and slot
                      ancestors identical; replaying the ancestors reproduces the run; the
                      ancestors visit the sorted particles in order
"""
from __future__ import annotations

import math

import numpy as np
import pytest

LOG_SQRT_2PI = 0.91893853320467274178


def _numpy_filter(N, rho, sig, mu, y, z, thr):
    rho, sig, mu = (float(np.float32(v)) for v in (rho, sig, mu))   # the oracle's config holds FP32
    stride = z.shape[1]
    sstat = math.sqrt(sig * sig / max(1.0 - rho * rho, 1e-6))
    h = mu + sstat * z[0, :N].astype(np.float64)
    prev_res, lse_prev, lwc = True, math.log(N), np.zeros(N)
    out = {"dll": [], "hmean": [], "ess": [], "resampled": [], "anc": np.zeros((len(y), N), dtype=np.int64)}
    for t in range(len(y)):
        if t > 0:
            h = mu + rho * (h - mu) + sig * z[t, :N].astype(np.float64)
        yt = float(y[t])
        lw = (0.0 if prev_res else lwc) + (-LOG_SQRT_2PI - 0.5 * yt * yt * np.exp(-h) - 0.5 * h)
        M = lw.max()
        e = np.exp(lw - M)
        S, Q = e.sum(), (e * e).sum()
        lse = M + math.log(S)
        out["dll"].append(lse - (math.log(N) if prev_res else lse_prev))
        out["hmean"].append((e * h).sum() / S)
        ess = S * S / Q
        out["ess"].append(ess)
        res = thr <= 0.0 or ess / N < thr
        out["resampled"].append(int(res))
        if res:
            order = np.lexsort((np.arange(N), h))
            cdf = np.cumsum(e[order])
            u = 0.5 * math.erfc(-float(z[t, stride - 4]) / math.sqrt(2.0))
            u23 = min(math.floor(u * 8388608.0), 8388607)
            targets = (u23 / 8388608.0 + np.arange(N)) * (cdf[-1] / N)
            j = np.minimum(np.searchsorted(cdf, targets, side="right"), N - 1)
            out["anc"][t] = order[j]
            h = h[order[j]]
            prev_res = True
        else:
            lwc, lse_prev, prev_res = lw, lse, False
    return out


@pytest.mark.parametrize("N,thr", [(1, 0.5), (7, 0.0), (64, 0.5), (301, 0.5), (512, 0.0)])
def test_noise_oracle_matches_numpy(orc, N, thr):
    T = 40
    rng = np.random.default_rng(N)
    stride = ((N + 3) & ~3) + 4
    z = rng.standard_normal((T, stride)).astype(np.float32)
    y = (np.exp(0.5 * rng.normal(-1.0, 0.5, T)) * rng.standard_normal(T)).astype(np.float32)
    o = orc.filter_noise_f64(N, 0.97, 0.15, -1.0, y, z, ess_threshold=thr)
    r = _numpy_filter(N, 0.97, 0.15, -1.0, y, z, thr)
    np.testing.assert_array_equal(o["resampled"], r["resampled"])
    for k in ("dll", "hmean", "ess"):
        np.testing.assert_allclose(o[k], r[k], rtol=1e-12, atol=1e-12)
    res = o["resampled"] == 1
    np.testing.assert_array_equal(o["anc"][res], r["anc"][res])
    rep = orc.filter_noise_f64(N, 0.97, 0.15, -1.0, y, z, ess_threshold=thr, anc_replay=o["anc"],
                               flags_replay=o["resampled"])
    np.testing.assert_array_equal(rep["dll"], o["dll"])
    np.testing.assert_array_equal(rep["hmean"], o["hmean"])


def test_noise_oracle_ancestors_follow_the_sorted_particles(orc):
    # with every tick resampling, the slot ancestors of tick t visit the particles of tick t in
    # ascending order of value
    N, T = 200, 12
    rng = np.random.default_rng(3)
    stride = ((N + 3) & ~3) + 4
    z = rng.standard_normal((T, stride)).astype(np.float32)
    y = rng.standard_normal(T).astype(np.float32)
    o = orc.filter_noise_f64(N, 0.9, 0.3, 0.0, y, z, ess_threshold=0.0)
    sstat = math.sqrt(0.09 / (1 - 0.81))
    h = 0.0 + sstat * z[0, :N].astype(np.float64)
    for t in range(T):
        if t > 0:
            h = 0.9 * h + 0.3 * z[t, :N].astype(np.float64)
        a = o["anc"][t]
        assert np.all(np.diff(h[a]) >= 0.0)
        h = h[a]
