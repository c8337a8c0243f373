"""CPU tests of the oracle's stage-by-stage restatement of the reference tick loop.

orc_ref_init / orc_ref_tick / orc_ref_resample are the stages of orc_ref_run exposed separately,
for the lock-step comparison with the reference run on a GPU. Chained single-threaded they must
reproduce orc_ref_run's per-tick (h_mean, loglik) bit for bit, and the state after init must be
the PCG32 state after draw 0 of every slot.
"""
from __future__ import annotations

import numpy as np
import pytest

RHO, SIG, MU = 0.97, 0.15, -1.0
PCG_A = 6364136223846793005


def _series(T, seed=42):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(ys, dtype=np.float32)


def test_init_state_is_draw_zero_stepped(orc):
    N, seed = 257, 42
    rng, h = orc.ref_init(N, RHO, SIG, MU, seed)
    for i in (0, 1, 128, 256):
        s0, inc = orc.pcg32_init(seed, i)
        assert int(rng[i, 1]) == inc
        assert int(rng[i, 0]) == (s0 * PCG_A + inc) % (1 << 64)
    assert np.all(np.isfinite(h))


@pytest.mark.parametrize("nu_obs", [0.0, 5.0])
def test_stages_chain_to_ref_run(orc, nu_obs):
    N, seed, T = 3000, 42, 25
    y = _series(T)
    hm_run, ll_run, cnt = orc.ref_run(N, RHO, SIG, MU, y, seed=seed, ess_threshold=0.0, nu_obs=nu_obs, nthreads=1)
    assert cnt == T
    rng, h = orc.ref_init(N, RHO, SIG, MU, seed)
    u23 = orc.host_u23_stream(seed, T)
    for t in range(T):
        hp, w, hm, ll, ess = orc.ref_tick(rng, h, RHO, SIG, MU, y[t], propagate=t > 0, nu_obs=nu_obs)
        assert hm == float(hm_run[t]) and ll == float(ll_run[t]), t
        assert 1.0 <= ess <= N
        u = np.float32(np.float32(u23[t]) * np.float32(1.0 / 8388608.0)) / np.float32(N)
        anc = orc.ref_resample(w, float(u))
        assert np.all(np.diff(anc) >= 0) and anc.min() >= 0 and anc.max() < N
        h = hp[anc]
