"""Source-level drop-in: the reference's own caller programs, compiled unchanged against this
repository's include/ (gpu_bpf.h, also answering to the reference header names gpu_bpf.cuh and
gpu_bpf_full.cuh) and linked to libgpubpf.so by oracle/build_ref.py (build_dropin), run on the GPU.

  bench_particle_scaling        tests/bench_particle_scaling.cu (gpu_bpf_step per tick, N 50K..1M),
                                built once as written and once with USE_PTX_FULL (gpu_bpf_full.cuh)
  test_cond_resample            tests/test_cond_resample.cu (ESS thresholds x scenarios at N=300K,
                                Silverman jitter written into the public state struct)
  test_bpf_matched_dgp          tests/test_bpf_matched_dgp.cu (nine matched-DGP scenarios against
                                EWMA and GARCH baselines, particle sweep, MC variance, throughput)
  test_mu_learning              smc2/test_mu_learning.cu (online mu / rho learning)
  bench_grad_overhead           tests/bench_grad_overhead.cu (cost of the learning score)

The programs print tables and assert nothing themselves; these tests read their output.
"""
from __future__ import annotations

import math
import os
import re
import subprocess
import sys

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

sys.path.insert(0, REPO)


def run_program(name, timeout=600):
    from oracle import build_ref
    path = build_ref.dropin_path(name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (build_ref.build_dropin needs the reference tree at build time)")
    out = subprocess.run([path], capture_output=True, text=True, timeout=timeout, cwd=os.path.dirname(path))
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert not re.search(r"\bnan\b", out.stdout, re.I), out.stdout[-3000:]
    return out.stdout


@pytest.mark.parametrize("name", ["bench_particle_scaling", "bench_particle_scaling_ptx_full"])
def test_bench_particle_scaling(name):
    text = run_program(name)
    rows = re.findall(r"^\s*(\d+)K\s+([\d.]+)ms\s+(\d+)\s+([\d.]+)us\s+(\d+) t/s", text, re.M)
    assert [int(r[0]) for r in rows] == [50, 100, 200, 300, 400, 500, 1000], text
    for _, ms, ticks, us, _tps in rows:
        assert int(ticks) == 1800
        assert 0.0 < float(us) < 1000.0 and math.isclose(float(ms) * 1e3 / 1800, float(us), rel_tol=0.02, abs_tol=0.1)


def test_cond_resample():
    text = run_program("test_cond_resample")
    # scenario tables: thresh | RMSE spkRMSE | resamp | rate | ms
    rows = re.findall(r"^\s*(always|[\d.]+)\s+│\s+([\d.]+)\s+([\d.]+)\s+│\s+(\d+)\s+│\s+([\d.]+)%", text, re.M)
    assert len(rows) == 20, text
    for thr, rmse, _spk, resamp, _rate in rows:
        assert 0.0 < float(rmse) < 2.0
        n = int(resamp)
        if thr == "always":
            assert n == 3000
        else:
            assert 0 < n < 3000
    # Silverman x threshold table: thresh silv | RMSE resamp%
    srows = re.findall(r"^\s*(always|0\.5)\s+(off|0\.3|0\.5|0\.7)\s+│\s+([\d.]+)\s+([\d.]+)%", text, re.M)
    assert len(srows) == 8, text
    for thr, _silv, rmse, pct in srows:
        assert 0.0 < float(rmse) < 2.0
        assert (float(pct) == 100.0) == (thr == "always")


def test_matched_dgp_suite():
    text = run_program("test_bpf_matched_dgp", timeout=1200)
    # TEST 1 rows: name | KF bound | BPF rmse bias ms | EWMA GARCH
    rows = re.findall(r"^\s*(.{18}) \|\s+([\d.]+) \|\s+([\d.]+)\s+[+-][\d.]+\s+\d+ms \|\s+([\d.]+)\s+([\d.]+)",
                      text, re.M)
    assert len(rows) == 9, text
    for name, _kf, bpf, ewma, garch in rows:
        assert float(bpf) < min(float(ewma), float(garch)), name


def test_mu_learning_program():
    text = run_program("test_mu_learning", timeout=900)
    assert "RMSE" in text or "rmse" in text


def test_grad_overhead_program():
    text = run_program("bench_grad_overhead", timeout=900)
    assert re.search(r"\d", text)
