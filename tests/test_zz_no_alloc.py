"""GPU test of gpu_bpf_run_static, the allocation-free entry point.

Callers that may not allocate device memory while they run (hosts with a
fixed start-up memory budget, latency-critical loops) use this entry point:
it keeps the whole filter in a fixed scratch area compiled into the library.
This test checks, through the C ABI, that two calls in a row give the same
records as the allocating path (gpu_bpf_create + gpu_bpf_step_many_device)
within the per-tick tolerance the other GPU tests use, and that a size above
the scratch capacity is rejected. The file name keeps it last in collection
order.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0
REC = 40   # sizeof(BpfTickRecord)


def _records(buf_u8):
    raw = buf_u8.cpu().numpy().tobytes()
    dt = np.dtype([("dloglik", "<f8"), ("loglik_ref", "<f8"), ("loglik_total", "<f8"),
                   ("h_mean", "<f4"), ("ess", "<f4"), ("resampled", "<i4"), ("tick", "<i4")])
    return np.frombuffer(raw, dtype=dt)


@pytest.mark.parametrize("n,thr,nu", [(100_000, 0.5, 0.0), (4096, 0.0, 5.0)])
def test_static_run_matches_allocating_path(bpf, n, thr, nu):
    import torch
    from gpubpf import _lib, dgp
    lib = bpf.load()
    T = 300
    _, ys = dgp.matched_series(T, RHO, SIG, MU, 7)
    y_dev = torch.tensor(np.asarray(ys, dtype=np.float32), device="cuda")

    ref_buf = torch.zeros(T * REC, dtype=torch.uint8, device="cuda")
    f = bpf.GpuBpf(n, RHO, SIG, MU, 0.0, nu, 11, ess_threshold=thr)
    f.step_many_device(y_dev.data_ptr(), T, ref_buf.data_ptr())
    torch.cuda.synchronize()
    f.close()
    ref = _records(ref_buf)

    for _ in range(2):     # two calls in a row share (and re-initialise) the scratch area
        buf = torch.zeros(T * REC, dtype=torch.uint8, device="cuda")
        rc = lib.gpu_bpf_run_static(n, RHO, SIG, MU, nu, 11, thr, y_dev.data_ptr(), T, buf.data_ptr(), None)
        assert rc == _lib.BPF_OK, rc
        torch.cuda.synchronize()
        got = _records(buf)
        np.testing.assert_array_equal(got["tick"], np.arange(T))
        np.testing.assert_array_equal(got["resampled"], ref["resampled"])
        assert np.max(np.abs(got["dloglik"] - ref["dloglik"])) <= 2e-4
        assert np.max(np.abs(got["h_mean"] - ref["h_mean"])) <= 2e-4
        assert np.max(np.abs(got["ess"] - ref["ess"]) / ref["ess"]) <= 1e-4
        assert abs(got["loglik_total"][-1] - ref["loglik_total"][-1]) <= 1e-4 * abs(ref["loglik_total"][-1])


def test_static_run_rejects_oversize(bpf):
    from gpubpf import _lib
    lib = bpf.load()
    rc = lib.gpu_bpf_run_static(_lib.BPF_STATIC_MAX_PARTICLES + 1, RHO, SIG, MU, 0.0, 1, 0.5, None, 0, None, None)
    assert rc == _lib.BPF_ERR_ARG
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
