"""The FP32 child-count estimate of the resampling kernels, checked on the host.

Pass 2 and the fused small-filter tick (bootstrap-particle-filter-in-ptx_b200/csrc/bpf_plain.cu)
count each parent's children from an FP32 estimate of the running count and trust it only when it
lies farther than an error bound from an integer; otherwise the element recounts in exact 64-bit
integers. The ancestors are bit-exact only if that bound is valid. The GPU parity tests check the
resulting ancestors on the data they run; here the kernels' FP32 operations, restated in C with the
same order and no contraction (oracle/bpf_oracle.c, orc_count_estimate_run), are driven over
millions of runs, adversarial ones included, and every estimate the bound declares safe must equal
the exact count. A bound shrunk on purpose must be caught.
"""
import numpy as np
import pytest

from oracle import oracle


@pytest.mark.parametrize("n", [16, 8, 4])          # pass 2's run per thread; the fused tick's chunks
@pytest.mark.parametrize("mode", [0, 1, 2])        # spread, on target boundaries, typical
def test_bound_never_trusts_a_wrong_estimate(n, mode):
    r = oracle.count_estimate_fuzz(seed=1000 + 10 * n + mode, n_runs=300_000, n=n, mode=mode)
    assert r["violations"] == 0, r
    assert r["safe"] > 0 and r["safe"] + r["recount"] == 300_000 * n


def test_typical_runs_rarely_recount():
    # a filter's resampling: uniform weights, about one target per weight
    r = oracle.count_estimate_fuzz(seed=5, n_runs=300_000, n=16, mode=2)
    assert r["violations"] == 0
    assert r["recount"] / (r["safe"] + r["recount"]) < 1e-3, r


@pytest.mark.parametrize("scale", [2.0 ** -12, 0.0])
def test_a_shrunk_bound_is_caught(scale):
    # the planted mistake: the kernels' bound scaled down; boundary runs must expose it
    r = oracle.count_estimate_fuzz(seed=77, n_runs=300_000, n=16, mode=1, bound_scale=scale)
    assert r["violations"] > 0, r


def test_exact_boundary_run():
    # sixteen weights of one half: the running sums are j/2 (units of 2^50); with the first target at
    # 3/2 and one every 1/2 the element sums land exactly on targets, so the estimate is either
    # recounted or right
    w = np.full(16, 0.5, dtype=np.float32)
    R0, D = 3 << 49, 1 << 49
    r = oracle.count_estimate_run(w, R0, D)
    assert r["violations"] == 0
    assert r["safe"] + r["recount"] == 16
    # weights that do not reach the first target have no children, estimated or recounted
    r = oracle.count_estimate_run(np.full(4, 2.0 ** -40, dtype=np.float32), 1 << 50, 1 << 50)
    assert r["violations"] == 0
