"""The reference's CUDA-C edition (gpu_bpf/gpu_bpf.cu behind gpu_bpf/gpu_bpf.cuh, the header this
build's C ABI replaces) run on the same GPU as a statistical checker: its noise is cuRAND XORWOW and
its Silverman jitter is switched off here (this build has none). Built into oracle/_ref/ by
oracle/build_ref.py; the tests skip when it was not built.

  plain filter, matched-DGP baseline scenario   RMSE of the filtered mean (T = 5000, N = 50000,
  (tests/test_bpf_matched_dgp.cu:181-189)        after 100 ticks) within 0.005 of the CUDA-C
                                                 edition's; resampling counts within 5%
  IMM, 8-model grid on a regime series           the reference's filters resampling every tick (its
  (gpu_bpf/gpu_bpf.cu:955-1080)                  IMM mixes BpfResult.log_lik, the log-evidence
                                                 since each filter's last resample; only then is that
                                                 the tick's increment, which this build mixes):
                                                 mixed-mean RMSE within 0.02, the most probable model
                                                 the same on >= 80% of ticks after 50, total log Z
                                                 within 10 nats (measured: 0.4827 / 0.4831, 94.4%,
                                                 0.08 nats)
  the reference's IMM in its default ESS mode    recounts earlier ticks' evidence: total log Z
                                                 far below the recursion's, model choice apart
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refc():
    from oracle import refgpu
    if not refgpu.available_cuda():
        pytest.skip("oracle/_ref/librefcuda.so not built (the reference tree was absent at build time)")
    refgpu.lib_cuda()
    return refgpu


def _rmse(hm, h, skip=100):
    e = np.asarray(hm[skip:], dtype=np.float64) - np.asarray(h[skip:], dtype=np.float64)
    return float(np.sqrt(np.mean(e * e)))


def test_plain_filter_against_cuda_edition(bpf, refc, golden):
    from gpubpf import dgp
    c = golden("dgp_scenarios.json")["scenarios"][0]             # Baseline (G/t5)
    h, y = dgp.matched_series(5000, c["rho"], c["sigma_z"], c["mu"], c["seed"], c["nu_state"], c["nu_obs"])
    y = np.asarray(y, dtype=np.float32)
    f = bpf.GpuBpf(50000, c["rho"], c["sigma_z"], c["mu"], c["nu_state"], c["nu_obs"], 142, ess_threshold=0.5)
    out = f.step_many(y.tolist())
    ours_n = f.state.resample_count
    f.close()
    ours = _rmse([r.h_mean for r in out], h)
    hm_r, _, ref_n = refc.cuda_run(50000, c["rho"], c["sigma_z"], c["mu"], y, c["nu_state"], c["nu_obs"], seed=142)
    ref = _rmse(hm_r, h)
    print(f"\n  baseline scenario: RMSE ours {ours:.4f} CUDA-C edition {ref:.4f}; resamples {ours_n} / {ref_n}")
    assert abs(ours - ref) <= 0.005
    assert abs(ours_n - ref_n) <= 0.05 * ref_n


def test_imm_against_cuda_edition(bpf, refc):
    from gpubpf import dgp, imm
    h, y = dgp.regime_series(1000, mus=(-1.5, -0.5), period=250, rho=0.97, sigma_z=0.2, seed=42)
    y = np.asarray(y, dtype=np.float32)
    models = imm.build_grid([0.95, 0.98], [0.1, 0.25], [-1.5, -0.5])
    assert len(models) == 8
    m = bpf.Imm(models, 4096, seed=42)
    hm, ll, best = [], [], []
    for v in y:
        r = m.step(float(v))
        hm.append(r.h_mean); ll.append(r.log_lik); best.append(r.best_model)
    m.close()
    hm_r, ll_r, best_r, _ = refc.cuda_imm_run(models, 4096, y, seed=42, ess_threshold=0.0)
    ours, ref = _rmse(hm, h, 50), _rmse(hm_r, h, 50)
    agree = float(np.mean(np.asarray(best[50:]) == best_r[50:]))
    dz = float(np.sum(np.asarray(ll, dtype=np.float64)) - np.sum(ll_r.astype(np.float64)))
    print(f"\n  IMM: mixed-mean RMSE ours {ours:.4f} CUDA-C edition {ref:.4f}; best model agrees on "
          f"{100 * agree:.1f}% of ticks; total log Z ours - reference {dz:+.2f}")
    assert abs(ours - ref) <= 0.02
    assert agree >= 0.8
    assert abs(dz) <= 10.0


def test_reference_imm_in_ess_mode_counts_past_evidence(bpf, refc):
    """With its default ESS threshold (0.5) the reference's IMM mixes each filter's log-evidence
    since its last resample, which counts earlier ticks again. Its model weights therefore leave the
    recursion on per-tick increments, the one this build (and the reference itself at threshold 0)
    computes. The log Z it reports per tick carries the recounted (negative) evidence: measured,
    the total falls 2180 nats below the recursion's and the most probable model agrees on about
    10% of ticks."""
    from gpubpf import dgp, imm
    _, y = dgp.regime_series(1000, mus=(-1.5, -0.5), period=250, rho=0.97, sigma_z=0.2, seed=42)
    y = np.asarray(y, dtype=np.float32)
    models = imm.build_grid([0.95, 0.98], [0.1, 0.25], [-1.5, -0.5])
    _, ll0, best0, _ = refc.cuda_imm_run(models, 4096, y, seed=42, ess_threshold=0.0)
    _, ll5, best5, _ = refc.cuda_imm_run(models, 4096, y, seed=42, ess_threshold=0.5)
    agree = float(np.mean(best0[50:] == best5[50:]))
    dz = float(np.sum(ll5.astype(np.float64)) - np.sum(ll0.astype(np.float64)))
    print(f"\n  reference IMM, threshold 0.5 vs 0: best model agrees on {100 * agree:.1f}% of ticks, "
          f"total log Z {dz:+.1f}")
    assert dz < -100.0
    assert agree < 0.5
