"""Allocation-failure injection (host side, no GPU fault): for every create path, each of its
device and pinned allocations in turn is made to fail (gpu_bpf_debug_fail_alloc), and the
create must return NULL with BPF_ERR_ALLOC and leave no allocation behind
(gpu_bpf_debug_live_allocs back to its value before the call)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

RHO, SIG, MU = 0.97, 0.15, -1.0


def _makers(bpf):
    from gpubpf import configs

    def plain():
        return bpf.GpuBpf(5000, RHO, SIG, MU, 0.0, 0.0, 3, ess_threshold=0.5)

    def plain_recording():
        f = bpf.GpuBpf(3000, RHO, SIG, MU, 0.0, 0.0, 3)
        try:
            f.record_ancestors(True)
        except BaseException:
            f.close()
            raise
        return f

    def apf():
        return bpf.GpuApf(5000, RHO, SIG, MU, 0.0, 0.0, 3)

    def imm():
        return bpf.Imm([{"rho": 0.97, "sigma_z": 0.15, "mu": m} for m in (-1.0, -0.5, 0.0)], 2048)

    def imm_plain_filters():
        return bpf.Imm([{"rho": 0.97, "sigma_z": 0.15, "mu": m} for m in (-1.0, 0.0)], 20000)

    def batch():
        return bpf.GpuBpfBatch(configs.config4(24), ess_threshold=0.5)

    def grad():
        return bpf.GradTape(4096, 50, checkpoint_every=8)

    def smc2():
        return bpf.Smc2(16, 256, 40, seed=2)

    def smc2_cpmmh():
        s = bpf.Smc2(16, 256, 40, seed=2)
        try:
            s.set_cpmmh_rho(0.9)
        except BaseException:
            s.close()
            raise
        return s

    return {"plain": plain, "plain_recording": plain_recording, "apf": apf, "imm": imm,
            "imm_plain_filters": imm_plain_filters, "batch": batch, "grad": grad, "smc2": smc2,
            "smc2_cpmmh": smc2_cpmmh}


@pytest.mark.parametrize("name", ["plain", "plain_recording", "apf", "imm", "imm_plain_filters", "batch", "grad",
                                  "smc2", "smc2_cpmmh"])
def test_create_cleans_up_after_a_failed_allocation(bpf, name):
    from gpubpf import _lib
    lib = bpf.load()
    make = _makers(bpf)[name]
    lib.gpu_bpf_debug_fail_alloc(-1)
    obj = make()                         # first use: per-device one-time set-up happens here
    obj.close()
    live0 = lib.gpu_bpf_debug_live_allocs()
    c0 = lib.gpu_bpf_debug_alloc_count()
    obj = make()
    n_alloc = lib.gpu_bpf_debug_alloc_count() - c0
    obj.close()
    assert lib.gpu_bpf_debug_live_allocs() == live0
    assert n_alloc >= 1
    try:
        for k in range(n_alloc):
            lib.gpu_bpf_debug_fail_alloc(k)
            with pytest.raises(bpf.BpfError) as e:
                make()
            assert e.value.code == _lib.BPF_ERR_ALLOC, (name, k, e.value.code)
            assert lib.gpu_bpf_debug_live_allocs() == live0, (name, k)
    finally:
        lib.gpu_bpf_debug_fail_alloc(-1)
    obj = make()                         # and the library still works afterwards
    obj.close()
    assert lib.gpu_bpf_debug_live_allocs() == live0
