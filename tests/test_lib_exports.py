"""CPU tests of the C ABI: the library builds for sm_100a, loads, exports every
symbol include/gpu_bpf.h declares, and validates arguments on the host before
any CUDA call (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from conftest import PKG_DIR, REPO

HEADER = os.path.join(REPO, "include", "gpu_bpf.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gpu_(?:bpf|imm|apf)_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bpf_build", os.path.join(PKG_DIR, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build_library()
    import gpubpf
    return gpubpf.load()


def test_header_declares_reference_api():
    names = header_functions()
    # gpu_bpf/gpu_bpf.cuh:56-85 and gpu_bpf_full.cuh:197-285
    for ref in ["gpu_bpf_create", "gpu_bpf_destroy", "gpu_bpf_step", "gpu_bpf_step_async",
                "gpu_bpf_get_result", "gpu_bpf_run_rmse", "gpu_bpf_set_bands", "gpu_bpf_set_adaptive_bands",
                "gpu_bpf_set_ess_threshold", "gpu_bpf_get_resample_count", "gpu_bpf_enable_mu_learning",
                "gpu_bpf_disable_mu_learning", "gpu_bpf_enable_rho_learning", "gpu_bpf_get_mu",
                "gpu_bpf_get_rho", "gpu_bpf_set_mu", "gpu_bpf_set_rho"]:
        assert ref in names


def test_every_declared_symbol_is_exported(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_binding_covers_header():
    from gpubpf import _lib
    assert set(header_functions()) <= set(_lib.SIGNATURES)


def test_result_layouts():
    from gpubpf import _lib
    assert C.sizeof(_lib.BpfResult) == 8
    assert C.sizeof(_lib.BpfTickRecord) == 40


def test_host_argument_validation(lib):
    from gpubpf import _lib
    bad = [
        (0, 0.97, 0.15, -1.0, 0.0, 0.0, 42),
        (-5, 0.97, 0.15, -1.0, 0.0, 0.0, 42),
        (4096, 1.0, 0.15, -1.0, 0.0, 0.0, 42),
        (4096, 0.97, 0.0, -1.0, 0.0, 0.0, 42),
        (4096, 0.97, -0.1, -1.0, 0.0, 0.0, 42),
        (4096, float("nan"), 0.15, -1.0, 0.0, 0.0, 42),
        (4096, 0.97, 0.15, float("inf"), 0.0, 0.0, 42),
        (4096, 0.97, 0.15, -1.0, 0.0, -1.0, 42),
        (4096, 0.97, 0.15, -1.0, 0.3, 0.0, 42),     # Student-t state noise needs round(nu_state) >= 1
    ]
    for args in bad:
        assert not lib.gpu_bpf_create(*args)
        assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
    s = lib.gpu_bpf_create(4096, 0.97, 0.15, -1.0, 5.0, 5.0, 42)   # Student-t state and observations
    if s:
        lib.gpu_bpf_destroy(s)
    else:
        assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_NODEVICE


def test_valid_create_without_gpu_fails_loudly(lib):
    from gpubpf import _lib
    s = lib.gpu_bpf_create(4096, 0.97, 0.15, -1.0, 0.0, 0.0, 42)
    if s:            # a GPU is present: the create must have worked
        lib.gpu_bpf_destroy(s)
        pytest.skip("GPU present")
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_NODEVICE


def test_null_state_calls_are_safe(lib):
    from gpubpf import _lib
    lib.gpu_bpf_destroy(None)
    r = lib.gpu_bpf_step(None, 0.1)
    assert r.h_mean != r.h_mean           # NaN
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_STATE
    assert lib.gpu_bpf_get_resample_count(None) == -1


def test_bands_only_identity(lib):
    from gpubpf import _lib
    one = (C.c_float * 1)(1.0)
    lib.gpu_bpf_set_bands(4096, 1, one, one)
    assert lib.gpu_bpf_last_error() == _lib.BPF_OK
    two = (C.c_float * 2)(0.5, 0.5)
    sc = (C.c_float * 2)(1.0, 3.0)
    lib.gpu_bpf_set_bands(4096, 2, two, sc)
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_UNSUPPORTED


def test_error_strings(lib):
    for code in range(8):
        assert lib.gpu_bpf_error_string(code)


def test_imm_host_side(lib):
    """gpu_imm_build_grid (host only) and gpu_imm_create's argument checks."""
    import ctypes as C
    from gpubpf import _lib, imm
    g = imm.build_grid([0.9, 0.97], [0.1, 0.2, 0.3], [-1.0, -0.5], nu_state=0.0, nu_obs=5.0)
    assert len(g) == 12
    assert [(round(m["rho"], 3), round(m["sigma_z"], 3), m["mu"]) for m in g[:3]] == \
        [(0.9, 0.1, -1.0), (0.9, 0.1, -0.5), (0.9, 0.2, -1.0)]             # rho-major, mu fastest
    assert all(m["nu_obs"] == 5.0 for m in g)
    models = (_lib.ImmModelParams * 65)()
    assert not lib.gpu_imm_create(models, 65, 1000, None, 1)               # IMM_MAX_MODELS = 64
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
    assert not lib.gpu_imm_create(models, 0, 1000, None, 1)
    assert lib.gpu_imm_get_prob(None, 0) == 0.0


def test_apf_host_side(lib):
    """gpu_apf_create's argument checks, NULL-state calls and the no-GPU failure."""
    from gpubpf import _lib
    for args in [(0, 0.97, 0.15, -1.0, 0.0, 0.0, 1), (4096, 1.0, 0.15, -1.0, 0.0, 0.0, 1),
                 (4096, 0.97, 0.0, -1.0, 0.0, 0.0, 1), (4096, 0.97, 0.15, -1.0, 0.3, 0.0, 1),
                 (4096, 0.97, 0.15, -1.0, 0.0, -2.0, 1), (4096, 0.97, 0.15, float("nan"), 0.0, 0.0, 1)]:
        assert not lib.gpu_apf_create(*args)
        assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
    lib.gpu_apf_destroy(None)
    r = lib.gpu_apf_step(None, 0.1)
    assert r.h_mean != r.h_mean
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_STATE
    assert lib.gpu_apf_get_loglik_total(None) != lib.gpu_apf_get_loglik_total(None)    # NaN
    s = lib.gpu_apf_create(4096, 0.97, 0.15, -1.0, 5.0, 5.0, 42)
    if s:
        lib.gpu_apf_destroy(s)
        pytest.skip("GPU present")
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_NODEVICE


def test_correlated_noise_and_smc2_host_side(lib):
    """The correlated-noise and SMC^2 entry points reject NULL handles and bad arguments on the
    host, before any CUDA call."""
    from gpubpf import _lib
    assert lib.gpu_bpf_smc2_set_cpmmh_rho(None, 0.5) == _lib.BPF_ERR_STATE
    assert lib.gpu_bpf_smc2_get_last_move(None, None, None, None, None, None) == _lib.BPF_ERR_STATE
    assert lib.gpu_bpf_smc2_get_noise(None, 0, 1, None) == _lib.BPF_ERR_STATE
    assert lib.gpu_bpf_batch_run_correlated(None, None, 1, None, None, 0.5, None, None, None) == _lib.BPF_ERR_STATE
    assert lib.gpu_bpf_batch_noise_offset(None, 0, 10) < 0
    assert not lib.gpu_bpf_smc2_create(1, 512, 100, None, 1)                 # fewer than 2 theta-particles
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
    assert not lib.gpu_bpf_smc2_create(64, 20000, 100, None, 1)              # above 16384 particles
    assert lib.gpu_bpf_last_error() == _lib.BPF_ERR_ARG
