"""Gradient form of the plain filter (include/gpu_bpf.h, "Gradient") and the
torch.autograd.Function over it.

The loss is the filter's total log-likelihood L(theta) = sum_t log p^(y_t | y_<t)
with the resampling ancestors held fixed: resampling indices carry no
gradient, resampled values do. This is the estimator of the reference's
tests/diff_bpf.py:186-237 (detached indices, :35-56 and :230-231), with two
stated differences: the stationary initial draw is differentiated too (it is
detached at :197-200) and there is no truncation window (:208-210 detaches
every 50 ticks). Tick 0 weights the initial particles without a prediction
step, as the plain filter does (gpu_bpf/gpu_bpf_ptx_full.cu:592).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import BpfError, BpfTickRecord, check


def ancestors_from_children(first_child: np.ndarray) -> np.ndarray:
    """Ancestor of every slot from the first-child list of a resampling tick."""
    f = np.asarray(first_child, dtype=np.int64)
    n = f.shape[0]
    counts = np.diff(np.append(f, n))
    return np.repeat(np.arange(n, dtype=np.int32), counts)


class GradTape:
    """Device tape of one taped forward run: child lists, checkpoints, normalisers."""

    def __init__(self, n_particles: int, max_ticks: int, checkpoint_every: int = 0, device=None):
        self._lib = _lib.load()
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        with torch.cuda.device(self.device):
            h = self._lib.gpu_bpf_grad_create(int(n_particles), int(max_ticks), int(checkpoint_every))
            if not h:
                raise BpfError(self._lib.gpu_bpf_last_error(), "gpu_bpf_grad_create")
            self._h = h
            self._stream = torch.cuda.ExternalStream(self._lib.gpu_bpf_grad_stream(h), device=self.device)
            # tape-owned buffers keep the captured graphs' pointers stable
            self._y = torch.zeros(int(max_ticks), dtype=torch.float32, device=self.device)
            self._ll = torch.zeros((), dtype=torch.float64, device=self.device)
            self._grad = torch.zeros(3, dtype=torch.float64, device=self.device)
            self._rep = torch.zeros(4, dtype=torch.float64, device=self.device)
        self.n_particles = int(n_particles)
        self.max_ticks = int(max_ticks)
        self.checkpoint_every = self._lib.gpu_bpf_grad_checkpoint_every(h)
        self.n_ticks = 0
        self.generation = 0
        self.theta = None

    @staticmethod
    def tape_bytes(n_particles: int, max_ticks: int, checkpoint_every: int = 0) -> int:
        return int(_lib.load().gpu_bpf_grad_tape_bytes(int(n_particles), int(max_ticks), int(checkpoint_every)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.gpu_bpf_grad_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> torch.cuda.ExternalStream:
        return self._stream

    def _enter(self):
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        self._stream.wait_event(ev)

    def _leave(self):
        ev = torch.cuda.Event()
        ev.record(self._stream)
        torch.cuda.current_stream(self.device).wait_event(ev)

    def forward(self, theta: Sequence[float], y: torch.Tensor, seed: int = 42, nu_obs: float = 0.0,
                nu_state: float = 0.0) -> torch.Tensor:
        """Taped run at theta = (mu, rho, sigma_z) on y (device float32): FP64 total loglik (0-d tensor)."""
        mu, rho, sig = (float(v) for v in theta)
        T = int(y.shape[0])
        if T > self.max_ticks:
            raise ValueError(f"{T} ticks exceed the tape's {self.max_ticks}")
        with torch.cuda.device(self.device):
            self._y[:T].copy_(y.reshape(-1).to(device=self.device, dtype=torch.float32))
            self._enter()
            check(self._lib.gpu_bpf_grad_forward(self._h, mu, rho, sig, float(nu_state), float(nu_obs), int(seed), 0.0,
                                                 C.c_void_p(self._y.data_ptr()), T, C.c_void_p(self._ll.data_ptr())),
                  "gpu_bpf_grad_forward")
            self._leave()
        self.n_ticks = T
        self.generation += 1
        self.theta = (mu, rho, sig)
        return self._ll.clone()

    def backward(self) -> torch.Tensor:
        """d loglik / d(mu, rho, sigma_z) of the last taped run (FP64, device)."""
        with torch.cuda.device(self.device):
            self._enter()
            check(self._lib.gpu_bpf_grad_backward(self._h, C.c_void_p(self._grad.data_ptr())), "gpu_bpf_grad_backward")
            self._leave()
        return self._grad.clone()

    def replay(self, theta: Sequence[float], per_tick: bool = False):
        """FP64 replay of the taped noise and ancestors at theta: tensor [loglik, dL/dmu, dL/drho, dL/dsigma]
        (and the per-tick [T, 4] values when per_tick)."""
        mu, rho, sig = (float(v) for v in theta)
        with torch.cuda.device(self.device):
            pt = torch.zeros((self.n_ticks, 4), dtype=torch.float64, device=self.device) if per_tick else None
            self._enter()
            check(self._lib.gpu_bpf_grad_replay(self._h, mu, rho, sig, C.c_void_p(self._rep.data_ptr()),
                                                C.c_void_p(pt.data_ptr()) if per_tick else None),
                  "gpu_bpf_grad_replay")
            self._leave()
        out = self._rep.clone()
        return (out, pt) if per_tick else out

    def fd_gradient(self, theta: Sequence[float], rel: float = 1e-3, points: int = 5) -> np.ndarray:
        """Central finite differences of the FP64 replay (common random numbers, the taped
        ancestors) with step rel*|theta_k|: the 5-point stencil (error O(h^4)) by default, or
        the 3-point one (O(h^2)). The log-likelihood is strongly curved in rho near 1, so at
        rel = 1e-3 the 3-point difference in rho is off by ~1e-3..1e-2 relative."""
        th = np.asarray(theta, dtype=np.float64)
        L = lambda t: float(self.replay(t)[0].item())
        out = np.zeros(3)
        for k in range(3):
            h = rel * abs(th[k])
            e = np.zeros(3)
            e[k] = h
            if points == 5:
                out[k] = (-L(th + 2 * e) + 8 * L(th + e) - 8 * L(th - e) + L(th - 2 * e)) / (12 * h)
            else:
                out[k] = (L(th + e) - L(th - e)) / (2 * h)
        return out

    def records(self):
        n = self.n_ticks
        arr = (BpfTickRecord * max(n, 1))()
        check(self._lib.gpu_bpf_grad_get_records(self._h, arr, n), "gpu_bpf_grad_get_records")
        return list(arr)[:n]

    def children(self, tick: int) -> np.ndarray:
        out = np.zeros(self.n_particles, dtype=np.int32)
        check(self._lib.gpu_bpf_grad_get_children(self._h, int(tick), out.ctypes.data_as(C.POINTER(C.c_int32))),
              "gpu_bpf_grad_get_children")
        return out

    def ancestors(self, tick: int) -> np.ndarray:
        """Ancestors (slots of tick `tick`) of the slots of tick `tick`+1."""
        return ancestors_from_children(self.children(tick))


class BpfLoglik(torch.autograd.Function):
    """loglik = BpfLoglik.apply(theta[3], y[T], tape, seed, nu_obs); backward = the adjoint kernel.

    theta = (mu, rho, sigma_z) in any float dtype on any device; the result is a
    0-d FP64 tensor on the tape's device.
    """

    @staticmethod
    def forward(ctx, theta, y, tape: GradTape, seed: int = 42, nu_obs: float = 0.0):
        th = theta.detach().to("cpu", torch.float64).tolist()
        ll = tape.forward(th, y, seed=seed, nu_obs=nu_obs)
        ctx.tape = tape
        ctx.generation = tape.generation
        ctx.theta_meta = (theta.dtype, theta.device)
        return ll

    @staticmethod
    def backward(ctx, grad_out):
        tape: GradTape = ctx.tape
        if tape.generation != ctx.generation:
            raise RuntimeError("the tape was overwritten by a later forward run before backward")
        g = tape.backward()
        dtype, device = ctx.theta_meta
        return (grad_out * g).to(device=device, dtype=dtype), None, None, None, None


_TAPES: dict = {}


def bpf_loglik(theta: torch.Tensor, y: torch.Tensor, n_particles: int, seed: int = 42, nu_obs: float = 0.0,
               tape: Optional[GradTape] = None, checkpoint_every: int = 0) -> torch.Tensor:
    """Differentiable FP64 total log-likelihood of the plain filter at theta = (mu, rho, sigma_z).

    A tape is created on first use for (device, n_particles, len(y)) and reused.
    """
    if tape is None:
        dev = y.device if y.is_cuda else torch.device("cuda", torch.cuda.current_device())
        key = (str(dev), int(n_particles), int(y.shape[0]), int(checkpoint_every))
        tape = _TAPES.get(key)
        if tape is None:
            tape = GradTape(n_particles, int(y.shape[0]), checkpoint_every, device=dev)
            _TAPES[key] = tape
    return BpfLoglik.apply(theta, y, tape, int(seed), float(nu_obs))


class BpfBatchLoglik(torch.autograd.Function):
    """loglik[B] = BpfBatchLoglik.apply(theta[B, 3], y[T], batch); backward: the batched adjoint.

    theta[b] = (mu, rho, sigma_z) of filter b of `batch` (a GpuBpfBatch that resamples every tick;
    its particle counts, seeds and observation models are kept). One gpu_bpf_batch_grad_run gives
    every filter's FP64 total log-likelihood and d loglik / d theta with the resampling ancestors
    held fixed (tests/diff_bpf.py:35-56 semantics), so backward only scales the stored gradient.
    """

    @staticmethod
    def forward(ctx, theta, y, batch):
        th = theta.detach().to("cpu", torch.float64)
        if th.dim() != 2 or th.shape[1] != 3 or th.shape[0] != batch.n_filters:
            raise ValueError(f"theta must have shape [{batch.n_filters}, 3]")
        batch.set_filters([dict(f, mu=float(m), rho=float(r), sigma_z=float(sg))
                           for f, (m, r, sg) in zip(batch.filters, th.tolist())])
        dev = y.device if y.is_cuda else torch.device("cuda", torch.cuda.current_device())
        y_d = y.detach().to(dev, torch.float32).contiguous()
        ll = torch.empty(batch.n_filters, dtype=torch.float64, device=dev)
        g = torch.empty(batch.n_filters, 3, dtype=torch.float64, device=dev)
        bs = torch.cuda.ExternalStream(batch.stream, device=dev)
        cur = torch.cuda.current_stream(dev)
        bs.wait_stream(cur)                       # inputs and outputs are ready before the run
        batch.grad_run(y_d.data_ptr(), int(y_d.shape[0]), ll.data_ptr(), g.data_ptr())
        cur.wait_stream(bs)                       # results are ready for the caller's stream
        y_d.record_stream(bs); ll.record_stream(bs); g.record_stream(bs)
        ctx.save_for_backward(g)
        ctx.theta_meta = (theta.dtype, theta.device)
        return ll

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        dtype, device = ctx.theta_meta
        return (grad_out.to(g.dtype)[:, None] * g).to(device=device, dtype=dtype), None, None


_BATCHES: dict = {}


def bpf_batch_loglik(theta: torch.Tensor, y: torch.Tensor, n_particles: Sequence[int],
                     seeds: Optional[Sequence[int]] = None, nu_obs: float = 0.0) -> torch.Tensor:
    """Differentiable FP64 total log-likelihoods loglik[B] of B plain filters at theta[B, 3] =
    (mu, rho, sigma_z), filter b with n_particles[b] (<= 16384) particles and seed seeds[b]
    (default 42 + b), resampling every tick. The batch is created on first use for
    (device, n_particles, seeds, nu_obs) and reused."""
    n = [int(v) for v in n_particles]
    sd = [42 + b for b in range(len(n))] if seeds is None else [int(v) for v in seeds]
    if len(sd) != len(n) or theta.shape[0] != len(n):
        raise ValueError("theta, n_particles and seeds must have the same length")
    dev = y.device if y.is_cuda else torch.device("cuda", torch.cuda.current_device())
    key = (str(dev), tuple(n), tuple(sd), float(nu_obs))
    batch = _BATCHES.get(key)
    if batch is None:
        from .batch import GpuBpfBatch
        th = theta.detach().to("cpu", torch.float64).tolist()
        with torch.cuda.device(dev):
            batch = GpuBpfBatch([{"mu": m, "rho": r, "sigma_z": s, "nu_obs": nu_obs, "n_particles": k, "seed": q}
                                 for (m, r, s), k, q in zip(th, n, sd)], ess_threshold=0.0)
        _BATCHES[key] = batch
    return BpfBatchLoglik.apply(theta, y, batch)

