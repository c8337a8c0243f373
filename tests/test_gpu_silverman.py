"""Silverman jitter after resampling (GpuBpfState.silverman_shrink > 0), the reference PTX
edition's option (gpu_bpf/gpu_bpf_ptx_full.cu:708-738, kernels ptx_assembly/bpf_kernels_full.ptx
:846-1060), against the FP64 oracle in lock step (ancestors and decisions replayed).

The jitter takes one draw from every particle slot's PCG32 stream, so the next propagation uses
the draw after it; the oracle restates that bookkeeping, so the particle clouds only stay
together if the device follows the same draw order. Tolerances as the plain filter's: per-tick
increment <= 2e-4 absolute, total <= 1e-4 relative, filtered mean <= 2e-4; particles after the
run <= 1e-4 absolute (FP32 against FP64).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


@pytest.mark.parametrize("N,thr,shrink", [(65536, 0.5, 0.5), (4097, 0.0, 0.7), (20000, 0.3, 0.3)])
def test_silverman_vs_fp64_oracle(bpf, orc, N, thr, shrink):
    from gpubpf import dgp
    T = 150
    _, ys = dgp.matched_series(T, RHO, SIG, MU, 7)
    y = np.asarray(ys, dtype=np.float32)
    f = bpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 5, ess_threshold=thr)
    f.state.silverman_shrink = shrink
    f.record_ancestors(True)
    o = orc.F64Filter(N, RHO, SIG, MU, seed=5, ess_threshold=thr, silverman=shrink)
    gd, od, gh, oh = [], [], [], []
    n_res = 0
    try:
        for t in range(T):
            f.step(float(y[t]))
            r = f.get_record()
            anc = np.frombuffer(f.get_ancestors()[1], dtype=np.int32) if r.resampled else None
            n_res += int(r.resampled)
            q = o.tick(y[t], anc=anc, flag=int(r.resampled))
            gd.append(r.dloglik); od.append(q["dll"]); gh.append(r.h_mean); oh.append(q["hmean"])
        hp = np.frombuffer(f.get_particles(), dtype=np.float32).astype(np.float64)
        op = o.particles()
    finally:
        f.close()
        o.close()
    gd, od = np.asarray(gd), np.asarray(od)
    assert n_res > 0
    assert np.max(np.abs(gd - od)) <= 2e-4, np.max(np.abs(gd - od))
    assert abs(gd.sum() - od.sum()) / abs(od.sum()) <= 1e-4
    assert np.max(np.abs(np.asarray(gh) - np.asarray(oh))) <= 2e-4
    assert np.max(np.abs(hp - op)) <= 1e-4, np.max(np.abs(hp - op))


def test_silverman_changes_the_cloud_and_graph_paths_agree(bpf):
    """The jitter moves the particles (against the same run without it), and the graph paths
    (step_many, single-tick graph) agree bit for bit with direct launches when it is on."""
    from gpubpf import dgp
    _, ys = dgp.matched_series(130, RHO, SIG, MU, 42)
    y = np.asarray(ys, dtype=np.float32)
    a = bpf.GpuBpf(8192, RHO, SIG, MU, seed=3, ess_threshold=0.5)
    b = bpf.GpuBpf(8192, RHO, SIG, MU, seed=3, ess_threshold=0.5)
    c = bpf.GpuBpf(8192, RHO, SIG, MU, seed=3, ess_threshold=0.5)
    for f in (a, b, c):
        f.state.silverman_shrink = 0.5
    ra = a.step_many(y.tolist(), records=True)
    rb = [b.step(float(v)) for v in y]
    for v in y:
        c.step_async(float(v))
    c.get_result()
    assert [r.h_mean for r in ra] == [r.h_mean for r in rb]
    assert bytes(a.get_particles()) == bytes(b.get_particles()) == bytes(c.get_particles())
    off = bpf.GpuBpf(8192, RHO, SIG, MU, seed=3, ess_threshold=0.5)
    ro = off.step_many(y.tolist(), records=True)
    assert any(x.h_mean != z.h_mean for x, z in zip(ra, ro))
    for f in (a, b, c, off):
        f.close()
