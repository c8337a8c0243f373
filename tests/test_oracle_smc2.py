"""CPU checks of the host restatement of the SMC^2 outer loop (oracle/smc2_outer.py) on
hand-made inputs: the PCG32 stream against its definition, the ESS and systematic resampling
against direct formulas, the random-walk proposal's covariance against numpy."""
from __future__ import annotations

import math

import numpy as np

from conftest import REPO  # noqa: F401  (puts the repository on sys.path)


def test_host_pcg_matches_definition():
    from oracle.smc2_outer import HostPcg, M64, PCG_A
    g = HostPcg(123, 0x5EED)
    inc = (0x5EED << 1) | 1
    st = 0
    st = (st * PCG_A + inc) & M64
    st = (st + 123) & M64
    st = (st * PCG_A + inc) & M64
    for _ in range(50):
        old = st
        st = (old * PCG_A + inc) & M64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        want = ((xs >> rot) | (xs << ((-rot) & 31))) & 0xFFFFFFFF
        assert g.next() == want
    u = [g.uniform() for _ in range(2000)]
    assert 0.0 < min(u) and max(u) < 1.0 and abs(np.mean(u) - 0.5) < 0.03


def test_ess_and_systematic_resampling():
    from oracle.smc2_outer import Smc2Outer
    o = Smc2Outer(8, 5)
    w = np.array([0.1, 2.0, 0.3, 0.05, 1.0, 0.2, 0.6, 0.4])
    o.logw = list(np.log(w))
    ess, _ = o.observe(np.zeros(8))
    assert math.isclose(ess, w.sum() ** 2 / (w ** 2).sum(), rel_tol=1e-12)
    rng_copy = Smc2Outer(8, 5).rng
    for _ in range(8 * 5):                       # the prior draws consume 5 uniforms per theta-particle
        rng_copy.next()
    idx = o.resample()
    u0 = rng_copy.uniform()
    cdf = np.cumsum(w / w.max())
    want = [min(int(np.searchsorted(cdf, (u0 + j) / 8 * cdf[-1], side="right")), 7) for j in range(8)]
    assert idx == want and o.logw == [0.0] * 8


def test_proposal_covariance():
    from oracle.smc2_outer import Smc2Outer
    o = Smc2Outer(400, 9)
    th = np.asarray(o.theta)
    diffs = []
    for _ in range(20):
        o.propose()
        diffs.append(np.asarray(o._pr) - np.asarray(o.theta))
    d = np.concatenate(diffs)
    want = 2.38 ** 2 / 3 * np.cov(th.T, bias=True)
    got = np.cov(d.T, bias=True)
    assert np.allclose(np.diag(got), np.diag(want), rtol=0.15)
