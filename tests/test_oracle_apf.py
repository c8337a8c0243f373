"""CPU tests of the oracle's auxiliary particle filter (orc_apf_f64) and of the recipe that
prepares the reference's PTX module for this GPU (oracle/build_ref.py).

  deterministic; tick 0 is a bootstrap tick (APF increment == the reference's value there)
  the APF and the bootstrap filter estimate the same log-likelihood and filtered mean
  (N = 20000, T = 120: |total loglik difference| < 0.5, mean |h_mean difference| < 0.05)
  replaying the ancestors is a pure function of them (identity anc reproduces a no-resampling path)
  the PTX retargeting drops non-ASCII bytes and rewrites exactly the .target line
"""
from __future__ import annotations

import numpy as np
import pytest

RHO, SIG, MU = 0.97, 0.15, -1.0


def _series(T, seed=42):
    from gpubpf import dgp
    h, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(h), np.asarray(ys, dtype=np.float32)


def test_apf_deterministic_and_tick0(orc):
    _, y = _series(30)
    a = orc.apf_f64(2000, RHO, SIG, MU, y, seed=5)
    b = orc.apf_f64(2000, RHO, SIG, MU, y, seed=5)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    assert a["dll"][0] == a["ll_ref"][0]                 # no first stage at tick 0
    assert np.all(np.isfinite(a["dll"])) and np.all(a["ess"] >= 1.0) and np.all(a["ess"] <= 2000)
    assert np.all(a["dll"][1:] != a["ll_ref"][1:])       # the first-stage term is present after tick 0


@pytest.mark.parametrize("nu_obs,nu_state", [(0.0, 0.0), (5.0, 0.0), (0.0, 5.0)])
def test_apf_agrees_with_bootstrap_filter(orc, nu_obs, nu_state):
    h, y = _series(120, seed=9)
    N = 20000
    a = orc.apf_f64(N, RHO, SIG, MU, y, seed=3, nu_obs=nu_obs, nu_state=nu_state)
    b = orc.filter_f64(N, RHO, SIG, MU, y, seed=3, ess_threshold=0.0, nu_obs=nu_obs, nu_state=nu_state)
    assert abs(a["dll"].sum() - b["dll"].sum()) < 0.5, (a["dll"].sum(), b["dll"].sum())
    assert np.mean(np.abs(a["hmean"] - b["hmean"])) < 0.05


def test_apf_replay_is_a_function_of_the_ancestors(orc):
    _, y = _series(20)
    N, T = 500, 20
    ident = np.tile(np.arange(N, dtype=np.int32), (T, 1))
    a = orc.apf_f64(N, RHO, SIG, MU, y, seed=1, anc1=ident, anc2=ident)
    b = orc.apf_f64(N, RHO, SIG, MU, y, seed=1, anc1=ident, anc2=ident)
    np.testing.assert_array_equal(a["dll"], b["dll"])
    c = orc.apf_f64(N, RHO, SIG, MU, y, seed=1)          # its own resampling: a different path
    assert not np.array_equal(a["hmean"], c["hmean"])


def test_reference_ptx_retarget():
    from oracle import build_ref
    src = ("// header ── box\n.version 8.8\n.target sm_120\n.address_size 64\n"
           "// comment é\n.visible .entry k() { ret; }\n").encode("utf-8")
    out = build_ref._retarget(src).decode("ascii")
    assert ".target sm_100a\n" in out and "sm_120" not in out
    assert all(ord(ch) < 128 for ch in out)
    assert ".visible .entry k() { ret; }" in out and ".version 8.8" in out
    with pytest.raises(RuntimeError):
        build_ref._retarget(b".version 8.8\n")
