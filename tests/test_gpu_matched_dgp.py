"""The reference's matched-DGP suite (tests/test_bpf_matched_dgp.cu) with assertions: the drop-in
filters the reference's own nine SV scenarios as well as the reference does.

The reference's suite prints tables and asserts nothing. Its inputs come from the golden fixture
tests/golden/dgp_scenarios.json (the scenarios' parameters and generator output, pinned against the
reference's generator by tests/test_oracle_golden.py); gpubpf.dgp regenerates the full series.

  test 1 (:449-483)    nine scenarios, T = 5000, N = 50000, filter seed 42 + 100 + i, RMSE of the
                       filtered mean against the true h after 100 ticks (gpu_bpf_run_rmse):
                       - within 0.005 of the reference's own GPU filter on the same series
                         (skipped when oracle/_ref is not built; measured: within 0.0011)
                       - below the EWMA(0.94) and best-GARCH(1,1) baselines of :320-395
                       - below the linearised-Kalman steady-state RMSE of :292-314 where that
                         model holds (Gaussian state noise; with t(5) state noise the filter's
                         RMSE exceeds it, 0.41 against 0.33 for the fast-reverting scenario, the
                         reference's own filter alike)
  test 2 (:489-518)    particle sweep on the Student-t scenario: RMSE does not grow with N
                       (beyond 0.003) and N = 256 is within 0.1 of N = 65536
  test 3 (:524-556)    ten filter seeds x 10000 particles: RMSE std below 0.01, mean within 0.01
                       of the N = 50000 run
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T, SKIP = 5000, 100


def _kalman_rmse(rho, sigma_z, nu_obs):
    """Linearised Kalman steady-state RMSE of test_bpf_matched_dgp.cu:292-314 (log y^2 observation
    noise variance pi^2/2, plus twice a trigamma-like term for Student-t observations)."""
    Q, a = sigma_z * sigma_z, rho * rho
    if nu_obs <= 0 or nu_obs > 100.0:
        R = 4.9348
    else:
        tg = 1.50 if nu_obs < 3.5 else 0.80 if nu_obs < 4.5 else 0.49 if nu_obs < 5.5 else 0.30 if nu_obs < 7.5 else 0.15
        R = 4.9348 + 2.0 * tg
    b = Q + R * (1.0 - a)
    c = -Q * R
    P = (-b + math.sqrt(b * b - 4.0 * a * c)) / (2.0 * a)
    return math.sqrt(P)


def _rmse(h_hat, h):
    e = np.asarray(h_hat[SKIP:], dtype=np.float64) - np.asarray(h[SKIP:], dtype=np.float64)
    return float(np.sqrt(np.mean(e * e)))


def _ewma_rmse(y, h, lam=0.94):
    """:320-345: h_hat = log of the EWMA variance before tick t's return."""
    y2 = np.asarray(y, dtype=np.float64) ** 2
    var = max(float(np.mean(y2[:min(len(y2), 20)])), 1e-10)
    hh = np.empty(len(y2))
    for t in range(len(y2)):
        hh[t] = math.log(var)
        var = max(lam * var + (1.0 - lam) * y2[t], 1e-10)
    return _rmse(hh, h)


def _garch_best_rmse(y, h):
    """:347-395: best RMSE of GARCH(1,1) over the reference's (alpha, beta) grid, omega by variance
    targeting."""
    y2 = np.asarray(y, dtype=np.float64) ** 2
    sv = float(np.mean(y2))
    best = 1e10
    for a in (0.02, 0.05, 0.08, 0.10, 0.15, 0.20):
        for b in (0.75, 0.80, 0.85, 0.90, 0.93, 0.95):
            if a + b >= 0.999:
                continue
            omega = sv * (1.0 - a - b)
            var = max(omega / (1.0 - a - b), 1e-10)
            hh = np.empty(len(y2))
            for t in range(len(y2)):
                hh[t] = math.log(var)
                var = max(omega + a * y2[t] + b * var, 1e-10)
            best = min(best, _rmse(hh, h))
    return best


@pytest.fixture(scope="module")
def scenarios(golden):
    from gpubpf import dgp
    g = golden("dgp_scenarios.json")
    out = []
    for c in g["scenarios"]:
        hs, ys = dgp.matched_series(T, c["rho"], c["sigma_z"], c["mu"], c["seed"], c["nu_state"], c["nu_obs"])
        out.append(dict(c, h=hs, y=ys))
    return out


def test_scenarios_full_comparison(bpf, scenarios):
    from oracle import refgpu
    have_ref = refgpu.available()
    rows = []
    for i, s in enumerate(scenarios):
        seed = 42 + 100 + i
        ours = bpf.run_rmse(s["y"], s["h"], 50000, s["rho"], s["sigma_z"], s["mu"], s["nu_state"], s["nu_obs"], seed)
        ref = None
        if have_ref:
            f = refgpu.RefGpuFilter(50000, s["rho"], s["sigma_z"], s["mu"], s["nu_state"], s["nu_obs"], seed=seed)
            hm, _ = f.run(np.asarray(s["y"], dtype=np.float32))
            f.close()
            ref = _rmse(hm, s["h"])
        kf = _kalman_rmse(s["rho"], s["sigma_z"], s["nu_obs"])
        ew = _ewma_rmse(s["y"], s["h"])
        ga = _garch_best_rmse(s["y"], s["h"])
        rows.append((s["name"], kf, ours, ref, ew, ga))
    print("\n  scenario            KF bound   ours     reference  EWMA94   GARCH")
    for name, kf, ours, ref, ew, ga in rows:
        print(f"  {name:18s}  {kf:7.4f}  {ours:7.4f}  {ref if ref is not None else float('nan'):9.4f}  {ew:7.4f}  {ga:7.4f}")
    for name, kf, ours, ref, ew, ga in rows:
        assert math.isfinite(ours), name
        if ref is not None:
            assert abs(ours - ref) <= 0.005, (name, ours, ref)
        assert ours < ew and ours < ga, (name, ours, ew, ga)
    for (name, kf, ours, _, _, _), s in zip(rows, scenarios):
        if s["nu_state"] == 0.0:
            assert ours < kf, (name, ours, kf)


def test_particle_sweep(bpf, scenarios):
    s = scenarios[1]                                   # Student-t (t5/t5), as the reference's sweep
    assert s["nu_state"] > 0 and s["nu_obs"] > 0
    res = {}
    for n in (256, 1024, 4096, 16384, 65536):
        res[n] = bpf.run_rmse(s["y"], s["h"], n, s["rho"], s["sigma_z"], s["mu"], s["nu_state"], s["nu_obs"], 42 + 400)
    print("\n  particle sweep:", {k: round(v, 4) for k, v in res.items()})
    ns = sorted(res)
    for a, b in zip(ns, ns[1:]):
        assert res[b] <= res[a] + 0.003, res
    assert res[256] - res[65536] < 0.1, res


def test_monte_carlo_variance(bpf, scenarios):
    s = scenarios[1]
    big = bpf.run_rmse(s["y"], s["h"], 50000, s["rho"], s["sigma_z"], s["mu"], s["nu_state"], s["nu_obs"], 42 + 101)
    v = np.array([bpf.run_rmse(s["y"], s["h"], 10000, s["rho"], s["sigma_z"], s["mu"], s["nu_state"], s["nu_obs"],
                               42 + 1000 + k * 137) for k in range(10)])
    print(f"\n  10 seeds x 10K: mean {v.mean():.4f} std {v.std():.4f}; 50K: {big:.4f}")
    assert v.std() < 0.01
    assert abs(v.mean() - big) < 0.01
