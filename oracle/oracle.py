"""ctypes face of the CPU oracle (oracle/bpf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by bench.py's CPU-baseline leg. The product never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "bpf_oracle.c")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")

CFLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-std=gnu11"]


def build(native: bool = False, force: bool = False) -> str:
    """Compile the oracle; native=True adds -march=native (timed baseline)."""
    out = os.path.join(BUILD, "liboracle_native.so" if native else "liboracle.so")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
        return out
    os.makedirs(BUILD, exist_ok=True)
    flags = list(CFLAGS)
    if native:
        flags[0] = "-O3"
        flags.append("-march=native")
    subprocess.run(["gcc", *flags, SRC, "-o", out + ".tmp", "-lm"], check=True)
    os.replace(out + ".tmp", out)
    return out


class OrcConfig(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int),
        ("rho", C.c_float), ("sigma_z", C.c_float), ("mu", C.c_float), ("nu_obs", C.c_float),
        ("seed", C.c_int),
        ("ess_threshold", C.c_float),
        ("nu_state", C.c_float),
        ("silverman", C.c_float),
    ]


_LIBS: dict = {}


def lib(native: bool = False) -> C.CDLL:
    key = bool(native)
    if key in _LIBS:
        return _LIBS[key]
    path = build(native=native)
    L = C.CDLL(path)
    u32, u64, i32, f32, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_float, C.c_double
    P = C.POINTER
    L.orc_pcg32_output.restype = u32; L.orc_pcg32_output.argtypes = [u64]
    L.orc_pcg32_init.restype = None; L.orc_pcg32_init.argtypes = [C.c_int, u32, P(u64), P(u64)]
    L.orc_pcg32_draw_stepped.restype = u32; L.orc_pcg32_draw_stepped.argtypes = [C.c_int, u32, C.c_int]
    L.orc_pcg32_draw_jump.restype = u32; L.orc_pcg32_draw_jump.argtypes = [C.c_int, u32, C.c_int]
    L.orc_pcg32_jump.restype = None; L.orc_pcg32_jump.argtypes = [u64, P(u64), P(u64)]
    L.orc_uniform.restype = f32; L.orc_uniform.argtypes = [u32]
    L.orc_host_pcg32.restype = u32; L.orc_host_pcg32.argtypes = [P(u64)]
    L.orc_host_seed.restype = u64; L.orc_host_seed.argtypes = [C.c_int]
    L.orc_acklam_f64.restype = f64; L.orc_acklam_f64.argtypes = [f64]
    L.orc_icdf_f64.restype = f64; L.orc_icdf_f64.argtypes = [f64]
    L.orc_acklam_f32.restype = f32; L.orc_acklam_f32.argtypes = [f32]
    L.orc_filter_f64.restype = C.c_int
    L.orc_filter_f64.argtypes = [P(OrcConfig), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_f64_create.restype = C.c_void_p; L.orc_f64_create.argtypes = [P(OrcConfig)]
    L.orc_f64_destroy.restype = None; L.orc_f64_destroy.argtypes = [C.c_void_p]
    L.orc_f64_tick.restype = C.c_int
    L.orc_f64_tick.argtypes = [C.c_void_p, f32, C.c_void_p, C.c_int, C.c_void_p]
    L.orc_f64_particles.restype = C.c_int; L.orc_f64_particles.argtypes = [C.c_void_p, C.c_void_p]
    L.orc_resample_fixed.restype = C.c_int
    L.orc_resample_fixed.argtypes = [C.c_int, C.c_void_p, C.c_void_p, u32, C.c_void_p]
    L.orc_ref_run.restype = C.c_int
    L.orc_ref_run.argtypes = [C.c_int, f32, f32, f32, f32, C.c_int, f32, C.c_void_p, C.c_int,
                              C.c_void_p, C.c_void_p, C.c_int, P(C.c_int)]
    L.orc_filter_noise_f64.restype = C.c_int
    L.orc_filter_noise_f64.argtypes = [P(OrcConfig), C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_apf_f64.restype = C.c_int
    L.orc_apf_f64.argtypes = [P(OrcConfig), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_ref_init.restype = C.c_int
    L.orc_ref_init.argtypes = [C.c_int, C.c_int, f32, f32, f32, C.c_void_p, C.c_void_p]
    L.orc_ref_tick.restype = C.c_int
    L.orc_ref_tick.argtypes = [C.c_int, C.c_void_p, C.c_void_p, f32, f32, f32, f32, f32, C.c_int, C.c_void_p,
                               C.c_void_p]
    L.orc_ref_resample.restype = C.c_int
    L.orc_ref_resample.argtypes = [C.c_int, C.c_void_p, f32, C.c_void_p]
    L.orc_num_threads.restype = C.c_int; L.orc_num_threads.argtypes = []
    L.orc_count_estimate_run.restype = C.c_longlong
    L.orc_count_estimate_run.argtypes = [P(f32), C.c_int, u64, u64, f32, P(C.c_longlong), P(C.c_longlong)]
    L.orc_count_estimate_fuzz.restype = None
    L.orc_count_estimate_fuzz.argtypes = [u64, C.c_longlong, C.c_int, C.c_int, f32, P(C.c_longlong)]
    L.orc_tstate_scale.restype = f64
    L.orc_tstate_scale.argtypes = [C.c_int, u32, C.c_int, C.c_int, f64]
    L.orc_grad_f64.restype = C.c_int
    L.orc_grad_f64.argtypes = [C.c_int, f64, f64, f64, f64, f64, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                               P(f64), C.c_void_p, C.c_void_p]
    _LIBS[key] = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def pcg32_draw(seed: int, i: int, t: int, stepped: bool = False) -> int:
    L = lib()
    return (L.orc_pcg32_draw_stepped if stepped else L.orc_pcg32_draw_jump)(seed, i, t)


def pcg32_init(seed: int, i: int):
    L = lib()
    s, inc = C.c_uint64(), C.c_uint64()
    L.orc_pcg32_init(seed, i, C.byref(s), C.byref(inc))
    return s.value, inc.value


def host_u23_stream(seed: int, n: int):
    L = lib()
    st = C.c_uint64(L.orc_host_seed(seed))
    return [L.orc_host_pcg32(C.byref(st)) >> 9 for _ in range(n)]


def filter_f64(n_particles, rho, sigma_z, mu, y, seed=42, ess_threshold=0.0, nu_obs=0.0,
               anc_replay=None, flags_replay=None, nu_state=0.0):
    """FP64 oracle run. Returns dict of per-tick arrays."""
    L = lib()
    y = np.ascontiguousarray(y, dtype=np.float32)
    T = y.shape[0]
    cfg = OrcConfig(int(n_particles), rho, sigma_z, mu, nu_obs, int(seed), ess_threshold, nu_state)
    out = {k: np.zeros(T, dtype=np.float64) for k in ("dll", "ll_ref", "hmean", "ess")}
    flags = np.zeros(T, dtype=np.int32)
    anc = None if anc_replay is None else np.ascontiguousarray(anc_replay, dtype=np.int32)
    fr = None if flags_replay is None else np.ascontiguousarray(flags_replay, dtype=np.int32)
    rc = L.orc_filter_f64(C.byref(cfg), _ptr(y), T, _ptr(anc), _ptr(fr), _ptr(out["dll"]), _ptr(out["ll_ref"]),
                          _ptr(out["hmean"]), _ptr(out["ess"]), _ptr(flags))
    if rc != 0:
        raise RuntimeError(f"orc_filter_f64 failed ({rc})")
    out["resampled"] = flags
    return out


class F64Filter:
    """The FP64 oracle filter stepped one tick at a time (orc_f64_*): follows a device run of any
    length in lock step, replaying each resampling tick's ancestors as it comes."""

    def __init__(self, n_particles, rho, sigma_z, mu, seed=42, ess_threshold=0.0, nu_obs=0.0, nu_state=0.0,
                 silverman=0.0):
        self._L = lib()
        self.N = int(n_particles)
        self._cfg = OrcConfig(self.N, rho, sigma_z, mu, nu_obs, int(seed), ess_threshold, nu_state, silverman)
        self._s = self._L.orc_f64_create(C.byref(self._cfg))
        if not self._s:
            raise MemoryError("orc_f64_create failed")

    def tick(self, y, anc=None, flag=None):
        """One tick; anc [N] int32 replays the ancestors if the tick resamples, flag replays the
        decision. Returns dict dll, ll_ref, hmean, ess, resampled."""
        a = None if anc is None else np.ascontiguousarray(anc, dtype=np.int32)
        if a is not None and a.shape[0] != self.N:
            raise ValueError("anc must hold N ancestors")
        out = np.zeros(5, dtype=np.float64)
        rc = self._L.orc_f64_tick(self._s, float(y), _ptr(a), -1 if flag is None else int(bool(flag)), _ptr(out))
        if rc != 0:
            raise RuntimeError(f"orc_f64_tick failed ({rc})")
        return {"dll": out[0], "ll_ref": out[1], "hmean": out[2], "ess": out[3], "resampled": int(out[4])}

    def particles(self):
        out = np.zeros(self.N, dtype=np.float64)
        self._L.orc_f64_particles(self._s, _ptr(out))
        return out

    def close(self):
        if self._s:
            self._L.orc_f64_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def filter_noise_f64(n_particles, rho, sigma_z, mu, y, z, ess_threshold=0.0, nu_obs=0.0, anc_replay=None,
                     flags_replay=None):
    """FP64 filter driven by the auxiliary noise z [T, stride] of a correlated-noise run (particles'
    normals in z[t, :N], the resampling normal in z[t, stride - 4]), sorting before every
    resampling. Returns dict of per-tick dll, hmean, ess, resampled and anc [T, N] (slot ancestors)."""
    L = lib()
    y = np.ascontiguousarray(y, dtype=np.float32)
    z = np.ascontiguousarray(z, dtype=np.float32)
    T = y.shape[0]
    assert z.shape[0] >= T
    N = int(n_particles)
    cfg = OrcConfig(N, rho, sigma_z, mu, nu_obs, 0, ess_threshold, 0.0)
    out = {k: np.zeros(T, dtype=np.float64) for k in ("dll", "hmean", "ess")}
    flags = np.zeros(T, dtype=np.int32)
    anc = np.zeros((T, N), dtype=np.int32)
    ar = None if anc_replay is None else np.ascontiguousarray(anc_replay, dtype=np.int32)
    fr = None if flags_replay is None else np.ascontiguousarray(flags_replay, dtype=np.int32)
    rc = L.orc_filter_noise_f64(C.byref(cfg), _ptr(y), T, _ptr(z), int(z.shape[1]), _ptr(ar), _ptr(fr),
                                _ptr(out["dll"]), _ptr(out["hmean"]), _ptr(out["ess"]), _ptr(flags), _ptr(anc))
    if rc != 0:
        raise RuntimeError(f"orc_filter_noise_f64 failed ({rc})")
    out["resampled"] = flags
    out["anc"] = anc
    return out


def apf_f64(n_particles, rho, sigma_z, mu, y, seed=42, nu_obs=0.0, nu_state=0.0, anc1=None, anc2=None):
    """FP64 auxiliary particle filter; anc1 / anc2 [T][N] replay the two stages' ancestors.
    Returns dict of per-tick arrays: dll (APF increment), ll_ref (the reference's log mean
    second-stage weight), hmean, ess."""
    L = lib()
    y = np.ascontiguousarray(y, dtype=np.float32)
    T = y.shape[0]
    cfg = OrcConfig(int(n_particles), rho, sigma_z, mu, nu_obs, int(seed), 0.0, nu_state)
    out = {k: np.zeros(T, dtype=np.float64) for k in ("dll", "ll_ref", "hmean", "ess")}
    a1 = None if anc1 is None else np.ascontiguousarray(anc1, dtype=np.int32)
    a2 = None if anc2 is None else np.ascontiguousarray(anc2, dtype=np.int32)
    rc = L.orc_apf_f64(C.byref(cfg), _ptr(y), T, _ptr(a1), _ptr(a2), _ptr(out["dll"]), _ptr(out["ll_ref"]),
                       _ptr(out["hmean"]), _ptr(out["ess"]))
    if rc != 0:
        raise RuntimeError(f"orc_apf_f64 failed ({rc})")
    return out


def count_estimate_fuzz(seed: int, n_runs: int, n: int, mode: int, bound_scale: float = 1.0) -> dict:
    """Host check of the resampling kernels' FP32 child-count estimate (orc_count_estimate_fuzz):
    n_runs random runs of n weights; mode 0 spread weights and spacings, 1 thresholds on target
    boundaries, 2 a filter's typical case. Returns the estimates declared safe that differ from
    the exact count ('violations'), and the safe and recounted element counts."""
    out = (C.c_longlong * 3)()
    lib().orc_count_estimate_fuzz(seed, n_runs, n, mode, bound_scale, out)
    return {"violations": out[0], "safe": out[1], "recount": out[2]}


def count_estimate_run(w, R0: int, D: int, bound_scale: float = 1.0) -> dict:
    """One run of weights w (FP32, in [0, 1], at most 16) against relative threshold R0 and spacing D."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    assert 1 <= w.size <= 16
    ns, nr = C.c_longlong(0), C.c_longlong(0)
    bad = lib().orc_count_estimate_run(w.ctypes.data_as(C.POINTER(C.c_float)), int(w.size), int(R0), int(D),
                                       bound_scale, C.byref(ns), C.byref(nr))
    return {"violations": bad, "safe": ns.value, "recount": nr.value}


def resample_fixed(w, tile_exp, u23):
    L = lib()
    w = np.ascontiguousarray(w, dtype=np.float32)
    te = np.ascontiguousarray(tile_exp, dtype=np.int32)
    anc = np.zeros(w.shape[0], dtype=np.int32)
    rc = L.orc_resample_fixed(int(w.shape[0]), _ptr(w), _ptr(te), int(u23), _ptr(anc))
    if rc != 0:
        raise RuntimeError(f"orc_resample_fixed failed ({rc})")
    return anc


def ref_run(n_particles, rho, sigma_z, mu, y, seed=42, ess_threshold=0.5, nu_obs=0.0, nthreads=0, native=False):
    """FP32 restatement of the reference tick loop: (hmean[T], loglik[T], resample_count)."""
    L = lib(native)
    y = np.ascontiguousarray(y, dtype=np.float32)
    T = y.shape[0]
    hm = np.zeros(T, dtype=np.float32)
    ll = np.zeros(T, dtype=np.float32)
    cnt = C.c_int(0)
    rc = L.orc_ref_run(int(n_particles), rho, sigma_z, mu, nu_obs, int(seed), ess_threshold, _ptr(y), T,
                       _ptr(hm), _ptr(ll), int(nthreads), C.byref(cnt))
    if rc != 0:
        raise RuntimeError(f"orc_ref_run failed ({rc})")
    return hm, ll, cnt.value


def ref_init(n_particles, rho, sigma_z, mu, seed=42):
    """The reference's initial state: (rng uint64 [N, 2] after draw 0, h0 float32 [N])."""
    L = lib()
    rng = np.zeros((int(n_particles), 2), dtype=np.uint64)
    h = np.zeros(int(n_particles), dtype=np.float32)
    rc = L.orc_ref_init(int(n_particles), int(seed), rho, sigma_z, mu, _ptr(rng), _ptr(h))
    if rc != 0:
        raise RuntimeError(f"orc_ref_init failed ({rc})")
    return rng, h


def ref_tick(rng, h, rho, sigma_z, mu, y, propagate=True, nu_obs=0.0):
    """One reference tick on given particles (FP32 restatement, stage by stage).

    rng: uint64 [N, 2] (state, inc), advanced in place when propagating; h: float32 [N] previous
    particles. Returns (propagated h, normalised w, h_mean, loglik, ess)."""
    L = lib()
    assert rng.dtype == np.uint64 and rng.flags.c_contiguous
    h = np.array(h, dtype=np.float32, copy=True)
    N = h.shape[0]
    w = np.zeros(N, dtype=np.float32)
    out = np.zeros(3, dtype=np.float32)
    rc = L.orc_ref_tick(N, _ptr(rng), _ptr(h), rho, sigma_z, mu, nu_obs, float(y), int(bool(propagate)), _ptr(w),
                        _ptr(out))
    if rc != 0:
        raise RuntimeError(f"orc_ref_tick failed ({rc})")
    return h, w, float(out[0]), float(out[1]), float(out[2])


def ref_resample(w, u):
    """The reference's systematic resampling (FP32 CDF, lower-bound search) with offset u = U/N."""
    L = lib()
    w = np.ascontiguousarray(w, dtype=np.float32)
    anc = np.zeros(w.shape[0], dtype=np.int32)
    rc = L.orc_ref_resample(int(w.shape[0]), _ptr(w), float(u), _ptr(anc))
    if rc != 0:
        raise RuntimeError(f"orc_ref_resample failed ({rc})")
    return anc


def grad_f64(n_particles, mu, rho, sigma_z, y, anc, seed=42, nu_obs=0.0, mode=1, nu_state=0.0):
    """FP64 loglik and d loglik / d(mu, rho, sigma_z) with ancestors anc[T][N] held fixed.

    mode 0 = forward-mode tangents, 1 = reverse-mode adjoint. Returns (ll, grad[3], dll[T]).
    """
    L = lib()
    y = np.ascontiguousarray(y, dtype=np.float32)
    T = y.shape[0]
    anc = np.ascontiguousarray(anc, dtype=np.int32).reshape(T, int(n_particles))
    ll = C.c_double(0.0)
    grad = np.zeros(3, dtype=np.float64)
    dll = np.zeros(T, dtype=np.float64)
    rc = L.orc_grad_f64(int(n_particles), float(mu), float(rho), float(sigma_z), float(nu_obs), float(nu_state),
                        int(seed), _ptr(y), T,
                        _ptr(anc), int(mode), C.byref(ll), _ptr(grad), _ptr(dll))
    if rc != 0:
        raise RuntimeError(f"orc_grad_f64 failed ({rc})")
    return ll.value, grad, dll


def num_threads(native: bool = False) -> int:
    return lib(native).orc_num_threads()
