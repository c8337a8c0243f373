"""GPU tests of the batched filter through the C ABI.

Parity contract: a batched filter computes the plain filter's per-particle
arithmetic and its fixed-point resampling, so for the same (theta, N, seed)
the ancestors of every tick and the final particles are bit-identical to a
plain filter's; log-likelihood increments differ only by the order of
floating-point sums (<= 2e-4 absolute per tick, <= 1e-6 relative in total).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAXN = 16384


def _series(T, seed=42, rho=0.97, sig=0.2, mu=-1.0):
    from gpubpf import dgp
    _, ys = dgp.matched_series(T, rho, sig, mu, seed)
    return np.asarray(ys, dtype=np.float32)


def _plain_reference(bpf, f, y, thr):
    """Plain filter with the batched filter's parameters: per-tick dll, ancestors, final particles."""
    n = f["n_particles"]
    p = bpf.GpuBpf(n, f["rho"], f["sigma_z"], f["mu"], 0.0, f.get("nu_obs", 0.0), f["seed"], ess_threshold=thr)
    p.record_ancestors(True)
    T = len(y)
    dll = np.zeros(T)
    anc = np.full((T, n), -1, dtype=np.int32)
    for t in range(T):
        p.step(float(y[t]))
        dll[t] = p.get_record().dloglik
        res, a = p.get_ancestors()
        if res:
            anc[t] = np.frombuffer(a, dtype=np.int32)
    h = np.frombuffer(p.get_particles(), dtype=np.float32).copy()
    p.close()
    return dll, anc, h


def _run_debug(bpf, filters, y, thr, threads=None):
    import torch
    B, T = len(filters), len(y)
    b = bpf.GpuBpfBatch(filters, ess_threshold=thr)
    if threads:
        for c, t in threads.items():
            b.set_threads(c, t)
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(B, dtype=torch.float64, device="cuda")
    dll = torch.zeros(B * T, dtype=torch.float64, device="cuda")
    anc = torch.full((B * T * MAXN,), -1, dtype=torch.int32, device="cuda")
    parts = torch.zeros(B * MAXN, dtype=torch.float32, device="cuda")
    b.run_debug(y_d.data_ptr(), T, ll.data_ptr(), dll.data_ptr(), anc.data_ptr(), parts.data_ptr())
    torch.cuda.synchronize()
    counts, hm = b.resample_counts()
    b.close()
    return (ll.cpu().numpy(), dll.cpu().numpy().reshape(B, T), anc.cpu().numpy().reshape(B, T, MAXN),
            parts.cpu().numpy().reshape(B, MAXN), counts)


FILTERS = [
    {"mu": -1.0, "rho": 0.97, "sigma_z": 0.15, "n_particles": 1, "seed": 3},
    {"mu": -0.5, "rho": 0.90, "sigma_z": 0.30, "n_particles": 100, "seed": 4},
    {"mu": -1.2, "rho": 0.99, "sigma_z": 0.10, "n_particles": 4096, "seed": 5},
    {"mu": -0.8, "rho": 0.95, "sigma_z": 0.25, "n_particles": 5000, "seed": 6},
    {"mu": -1.5, "rho": 0.85, "sigma_z": 0.40, "n_particles": 9000, "seed": 7},
    {"mu": -1.0, "rho": 0.97, "sigma_z": 0.20, "n_particles": 16384, "seed": 8},
]


@pytest.mark.parametrize("thr", [0.0, 0.5])
def test_batch_matches_plain_filter(bpf, thr):
    y = _series(40)
    ll, dll, anc, parts, counts = _run_debug(bpf, FILTERS, y, thr)
    for b, f in enumerate(FILTERS):
        n = f["n_particles"]
        p_dll, p_anc, p_h = _plain_reference(bpf, f, y, thr)
        assert np.max(np.abs(dll[b] - p_dll)) <= 2e-4, b
        assert abs(ll[b] - p_dll.sum()) <= 1e-6 * max(1.0, abs(p_dll.sum())), b
        resampled = p_anc[:, 0] >= 0
        assert counts[b] == int(resampled.sum())
        for t in np.nonzero(resampled)[0]:
            np.testing.assert_array_equal(anc[b, t, :n], p_anc[t], err_msg=f"filter {b} tick {t}")
        np.testing.assert_array_equal(parts[b, :n], p_h, err_msg=f"filter {b} particles")


def test_batch_student_t(bpf):
    fl = [dict(f, nu_obs=5.0) for f in FILTERS[2:5]]
    y = _series(30, seed=3)
    ll, dll, anc, parts, _ = _run_debug(bpf, fl, y, 0.0)
    for b, f in enumerate(fl):
        p_dll, p_anc, p_h = _plain_reference(bpf, f, y, 0.0)
        assert np.max(np.abs(dll[b] - p_dll)) <= 2e-4
        np.testing.assert_array_equal(parts[b, :f["n_particles"]], p_h)


def test_batch_vs_fp64_oracle(bpf, orc):
    y = _series(80, seed=7)
    fl = FILTERS[2:4]
    ll, dll, anc, parts, _ = _run_debug(bpf, fl, y, 0.0)
    for b, f in enumerate(fl):
        n = f["n_particles"]
        o = orc.filter_f64(n, f["rho"], f["sigma_z"], f["mu"], y, seed=f["seed"], ess_threshold=0.0,
                           anc_replay=anc[b, :, :n], flags_replay=np.ones(len(y), dtype=np.int32))
        assert abs(ll[b] - o["dll"].sum()) <= 1e-4 * abs(o["dll"].sum())
        assert np.max(np.abs(dll[b] - o["dll"])) <= 2e-4


def test_batch_cta_shape_does_not_change_results(bpf):
    y = _series(25)
    fl = FILTERS[1:]
    a = _run_debug(bpf, fl, y, 0.5, threads={0: 64, 2: 128, 3: 256, 4: 512})
    b = _run_debug(bpf, fl, y, 0.5, threads={0: 256, 2: 512, 3: 1024, 4: 1024})
    np.testing.assert_array_equal(a[2], b[2])          # ancestors
    np.testing.assert_array_equal(a[3], b[3])          # particles
    # log-likelihood: the per-thread FP32 partial sums take other particles under another CTA
    # shape (FP32 rounding of S, sum W^2, sum W h), so totals agree to about 1e-8 relative
    np.testing.assert_allclose(a[0], b[0], rtol=1e-7)


def test_batch_graph_run_and_autotune(bpf, tmp_path):
    import torch
    from gpubpf import configs
    fl = configs.batch_thetas(48)
    y = _series(50)
    b = bpf.GpuBpfBatch(fl, ess_threshold=0.0)
    ll_host, hm = b.run(y.tolist())
    y_d = torch.tensor(y, device="cuda")
    ll = torch.zeros(len(fl), dtype=torch.float64, device="cuda")
    for _ in range(2):                                  # graph built once, replayed
        b.run_device(y_d.data_ptr(), len(y), ll.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_allclose(ll.cpu().numpy(), ll_host, rtol=0, atol=0)
    cache = str(tmp_path / "tune.txt")
    b.autotune(y[:20].tolist(), cache_path=cache)
    chosen = [b.get_threads(c) for c in range(5)]
    assert all(t in (64, 128, 256, 512, 1024) for t in chosen)
    ll2, _ = b.run(y.tolist())
    np.testing.assert_allclose(ll2, ll_host, rtol=1e-7)  # the autotuned shapes regroup the FP32 partials
    lines = open(cache).read().split()
    assert len(lines) % 3 == 0 and len(lines) >= 3
    b2 = bpf.GpuBpfBatch(fl, ess_threshold=0.0)
    b2.autotune(y[:20].tolist(), cache_path=cache)      # served from the cache
    assert [b2.get_threads(c) for c in range(5)] == chosen
    b.close(); b2.close()
