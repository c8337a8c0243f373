"""Checkpoint / resume of the plain filter (gpu_bpf_save / gpu_bpf_load): a filter restored from
a checkpoint continues bit for bit as the saved one does (records, particles, running
log-likelihood), whatever filter it is loaded into, including mid-run with carried weights
(ESS-skipped ticks), Student-t noises, Silverman jitter and the fused small-filter path."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def _y(T, seed=7):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, RHO, SIG, MU, seed)
    return np.asarray(ys, dtype=np.float32)


def _key(recs):
    return [(r.dloglik, r.loglik_ref, r.loglik_total, r.h_mean, r.ess, r.resampled, r.tick) for r in recs]


@pytest.mark.parametrize("N,thr,nu_obs,nu_state,silv", [(20000, 0.5, 0.0, 0.0, 0.0), (4096, 0.5, 5.0, 5.0, 0.0),
                                                        (9000, 0.3, 0.0, 0.0, 0.5), (70000, 0.0, 5.0, 0.0, 0.0)])
def test_resume_is_bit_identical(bpf, N, thr, nu_obs, nu_state, silv):
    y = _y(150)
    a = bpf.GpuBpf(N, RHO, SIG, MU, nu_state, nu_obs, 31, ess_threshold=thr)
    a.state.silverman_shrink = silv
    a.step_many(y[:83].tolist())
    blob = a.save()
    rest_a = a.step_many(y[83:].tolist(), records=True)
    parts_a = bytes(a.get_particles())
    total_a = a.get_loglik_total()
    count_a = a.get_resample_count()
    a.close()

    b = bpf.GpuBpf(N, 0.9, 0.3, 0.0, 0.0, 0.0, 5, ess_threshold=0.9)   # other parameters, overwritten
    b.step_many(y[:10].tolist())
    b.load(blob)
    assert b.state.rho == np.float32(RHO) and b.state.ess_threshold == np.float32(thr)
    assert b.state.silverman_shrink == np.float32(silv) and b.state.timestep == 83
    rest_b = []
    for v in y[83:]:
        b.step(float(v))
        rest_b.append(b.get_record())
    assert _key(rest_a) == _key(rest_b)
    assert bytes(b.get_particles()) == parts_a
    assert b.get_loglik_total() == total_a and b.get_resample_count() == count_a
    b.close()


def test_load_rejects_mismatched_checkpoints(bpf):
    from gpubpf import _lib
    a = bpf.GpuBpf(5000, RHO, SIG, MU, seed=1)
    a.step_many(_y(20).tolist())
    blob = a.save()
    b = bpf.GpuBpf(6000, RHO, SIG, MU, seed=1)
    with pytest.raises(bpf.BpfError) as e:
        b.load(blob)
    assert e.value.code == _lib.BPF_ERR_ARG
    bad = bytearray(blob)
    bad[0] ^= 0xFF
    with pytest.raises(bpf.BpfError) as e:
        a.load(bytes(bad))
    assert e.value.code == _lib.BPF_ERR_ARG
    with pytest.raises(bpf.BpfError) as e:
        a.load(blob[:100])
    assert e.value.code == _lib.BPF_ERR_ARG
    a.load(blob)                                   # the untouched checkpoint still loads
    a.close(); b.close()
