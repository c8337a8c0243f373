#!/usr/bin/env python3
"""Benchmark: plain SV bootstrap particle filter, particle-steps/s.

Workload (the reference's headline scaling configuration, at its target size):
SV model mu=-1.0, phi=0.97, sigma_eta=0.15; observations from the matched DGP
with seed 7 (T=5000); N=2^24 particles; resample when ESS < 0.5 N. One step =
one filter pass over the T=5000 series (re-seed + 5000 ticks).

  value  device-resident run: y already in HBM, ticks replayed as a CUDA graph
  e2e    the same run through gpu_bpf_step_many with host buffers (pinned
         staging, H2D of y and D2H of the per-tick records inside the timing)
  roofline  pass-1 / pass-2 kernel durations from CUDA events on the filter
         stream during a profiled pass of the same workload
  cpu_baseline  FP32 restatement of the reference tick loop (oracle/), OpenMP
         over all host cores, on a bounded number of ticks of the same run
  sweep     the scaling sweep N = 2^16 .. 51.2M (first 1000 ticks, ESS<0.5N)
  config1   N=4096, T=1000, always resample: GPU and the CPU restatement on 1
         core and all cores, loglik against the FP64 oracle
  batched   1024 filters with their own theta and N (512..16384), T=2000, one
         persistent launch per size class in one CUDA graph, against the plain
         filter run per filter
  gradient  d loglik / d theta at N=2^20, T=2000 (taped forward + adjoint
         backward) against the plain forward, with the full-size FP64 replay and
         finite-difference checks
  batch_gradient  forward + backward of 256 filters x 8192 particles over a
         4000-tick regime-switching series, against the batched forward
  extensions  Student-t noise, online learning, the auxiliary particle filter,
         IMM and SMC^2, each on its own small workload (bench_extensions)

`--impl reference` times that CPU restatement alone (rank 0) and prints the
same metric; when oracle/_ref holds the reference's own GPU filter (built from
the reference sources) its line adds `reference_gpu`, that filter timed on this
GPU on the same workload. Multi-GPU (torchrun): independent replicas, one per GPU, seeds
differ per rank; no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(REPO, "bootstrap-particle-filter-in-ptx_b200")
for _p in (REPO, PKG_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

RHO, SIG, MU = 0.97, 0.15, -1.0
DEVSTATE_BYTES = 200          # sizeof(bpf::DevState), read back once after a host-buffer run
RECORD_BYTES = 40             # sizeof(BpfTickRecord)
L2_NOTE = "working set h 4B + w 4B per particle = 128 MiB per tick at N=2^24 (> 126 MB L2); 256 MiB L2 flush between steps"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1 << 24)
    ap.add_argument("--ticks", type=int, default=5000)
    ap.add_argument("--ess", type=float, default=0.5)
    ap.add_argument("--dgp-seed", type=int, default=7)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-filters", type=int, default=1024)
    ap.add_argument("--batch-ticks", type=int, default=2000)
    ap.add_argument("--no-gradient", action="store_true")
    ap.add_argument("--grad-n", type=int, default=1 << 20)
    ap.add_argument("--grad-ticks", type=int, default=2000)
    ap.add_argument("--no-batch-gradient", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--sweep-ticks", type=int, default=1000)
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--no-extensions", action="store_true")
    ap.add_argument("--bgrad-filters", type=int, default=256)
    ap.add_argument("--bgrad-ticks", type=int, default=4000)
    ap.add_argument("--parity-ticks", type=int, default=20,
                    help="ticks of the headline run followed by the FP64 oracle in lock step (0 = off)")
    ap.add_argument("--plumbing-check", action="store_true",
                    help="CPU-only check of the multi-rank path (gloo): rank launch, shard, gather, max-reduce")
    ap.add_argument("--smc2-only", type=int, default=0, metavar="UPDATES",
                    help="run only the SMC^2 workload of the extensions (50 warm-up updates, then UPDATES timed "
                         "ones; for a kernel launch list of one update) and print its line")
    return ap.parse_args()


FALLBACK_HBM_GBS = 6650.0   # an earlier STREAM-style copy measurement on this pool's B200s


def load_peaks():
    """(HBM GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json when it holds a
    usable `hbm_gbs`, else the fallback figure."""
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        if v > 0.0:
            return v, "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return FALLBACK_HBM_GBS, f"fallback {FALLBACK_HBM_GBS:.0f} GB/s (MEASURED_PEAKS.json absent or without hbm_gbs)"


def load_traffic():
    """Per-launch DRAM bytes per particle from the committed ncu summary, if any."""
    p = os.path.join(REPO, "profiles", "ncu_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            parts = line.split()
            if len(parts) >= 3 and parts[1] == "dram_bytes_per_particle":
                out[parts[0]] = float(parts[2])
    return out


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1])); mx.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(n, y, ess, seconds, native=True):
    """FP32 restatement of the reference tick loop on all host cores, bounded sample."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    oracle.lib(native)
    t0 = time.perf_counter()
    oracle.ref_run(n, RHO, SIG, MU, y[:2], seed=42, ess_threshold=ess, nthreads=cores, native=native)
    per_tick = max((time.perf_counter() - t0) / 2.0, 1e-6)
    ticks = int(max(2, min(len(y), seconds / per_tick)))
    t0 = time.perf_counter()
    oracle.ref_run(n, RHO, SIG, MU, y[:ticks], seed=42, ess_threshold=ess, nthreads=cores, native=native)
    dt = time.perf_counter() - t0
    return {"value": n * ticks / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"N={n}, first {ticks} ticks of the DGP-seed-7 series, ESS<{ess}N; oracle/bpf_oracle.c "
                      f"orc_ref_run (FP32 reference tick loop, OpenMP {cores} threads, -O3 -march=native)",
            "us_per_tick": dt / ticks * 1e6}


def bench_batched(dev, args, lib, rank, world, barrier):
    """Configuration 4: B=1024 filters, theta and N drawn as in gpubpf.configs, T=2000 ticks of one
    series (mu=-1, phi=0.97, sigma_eta=0.2, DGP seed 42), resampling every tick. Filters are sharded
    across ranks by LPT on N. Comparator: the plain filter run per filter, each replaying its own
    CUDA graph on its own stream (all concurrent), on every 16th filter of this rank's shard."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import gpubpf
    from gpubpf import configs, dgp, parallel
    B, T = args.batch_filters, args.batch_ticks
    allf = configs.config4(B)
    idx, fl = parallel.shard(allf, rank, world)
    _, ys = dgp.matched_series(T, 0.97, 0.2, -1.0, 42)
    y = np.asarray(ys, dtype=np.float32)
    y_d = torch.tensor(y, device=dev)
    steps_local = float(sum(f["n_particles"] for f in fl)) * T
    steps_total = float(sum(f["n_particles"] for f in allf)) * T
    b = gpubpf.GpuBpfBatch(fl, ess_threshold=0.0)
    b.autotune(y[:64].tolist())
    shapes = [b.get_threads(c) for c in range(5)]
    ll = torch.zeros(len(fl), dtype=torch.float64, device=dev)
    bs = torch.cuda.ExternalStream(b.stream, device=dev)
    for _ in range(3):
        b.run_device(y_d.data_ptr(), T, ll.data_ptr())
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = max(1, args.steps)
    e0.record(bs)
    for _ in range(reps):
        b.run_device(y_d.data_ptr(), T, ll.data_ptr())
    e1.record(bs)
    barrier()
    ms = torch.tensor([e0.elapsed_time(e1) / reps], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms = float(ms.item())
    value = steps_total / (ms / 1e3)
    finite = bool(torch.isfinite(ll).all().item())
    b.close()

    # several ranks: every filter's log-likelihood gathered from the shards must equal one GPU running
    # all filters (both with the default CTA shapes: a filter's result depends on its class's shape,
    # never on the other filters in the launch)
    shard_check = None
    if world > 1:
        bd = gpubpf.GpuBpfBatch(fl, ess_threshold=0.0)
        ll_d = torch.zeros(len(fl), dtype=torch.float64, device=dev)
        bd.run_device(y_d.data_ptr(), T, ll_d.data_ptr())
        torch.cuda.synchronize(dev)
        bd.close()
        full = parallel.gather_results(idx, ll_d.cpu().tolist(), B)
        if rank == 0:
            ba = gpubpf.GpuBpfBatch(allf, ess_threshold=0.0)
            ll_a = torch.zeros(B, dtype=torch.float64, device=dev)
            ba.run_device(y_d.data_ptr(), T, ll_a.data_ptr())
            one = ll_a.cpu().tolist()
            ba.close()
            diffs = [abs(a - b_) for a, b_ in zip(full, one)]
            shard_check = {"filters": B, "ranks": world, "bit_identical": all(a == b_ for a, b_ in zip(full, one)),
                           "max_abs_diff": max(diffs),
                           "method": "per-filter loglik gathered from the LPT shards vs one GPU running all filters"}

    # comparator: per-filter plain launches (graph per filter, one stream each)
    sub = fl[::16]
    filt = [gpubpf.GpuBpf(f["n_particles"], f["rho"], f["sigma_z"], f["mu"], 0.0, 0.0, f["seed"], ess_threshold=0.0)
            for f in sub]
    recs = [torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev) for _ in sub]
    for g, r in zip(filt, recs):
        g.step_many_device(y_d.data_ptr(), T, r.data_ptr())      # builds each filter's graph
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for g, f, r in zip(filt, sub, recs):
        g.reset(f["seed"])
        g.step_many_device(y_d.data_ptr(), T, r.data_ptr())
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    per_filter = float(sum(f["n_particles"] for f in sub)) * T / dt
    for g in filt:
        g.close()
    return {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "ms_per_run": ms, "filters": B, "ticks": T, "particle_steps_per_run": steps_total,
            "shard": f"LPT on N over {world} rank(s)", "cta_threads_per_class": shapes,
            "per_filter_plain": {"value": per_filter, "unit": "particle-steps/s", "filters_timed": len(sub),
                                 "method": "gpu_bpf_step_many_device per filter, own stream, CUDA graph"},
            "speedup_vs_per_filter": value / per_filter if world == 1 else None,
            "loglik_finite": finite, "shard_check": shard_check}


def bench_sweep(dev, args, lib, rank, world, barrier):
    """Configuration 2 scaling sweep: N in {2^16, 2^18, 2^20, 2^22, 2^24, 51,200,000}, same theta and DGP
    seed 7, ESS<0.5N, the first --sweep-ticks ticks of the T=5000 series. Device-resident runs (one CUDA
    graph each), CUDA events on the filter stream, 3 warm-ups, mean of --steps runs, max over ranks.
    HBM fraction = algorithmic bytes (pass 1 12 B/particle, +4 on carry ticks; pass 2 12 B/particle on
    resampling ticks) / run time / measured peak."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import gpubpf
    from gpubpf import dgp
    T = args.sweep_ticks
    _, ys = dgp.matched_series(5000, RHO, SIG, MU, args.dgp_seed)
    y = torch.tensor(np.asarray(ys[:T], dtype=np.float32), device=dev)
    rec = torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev)
    peak, _ = load_peaks()
    out = []
    for N in (1 << 16, 1 << 18, 1 << 20, 1 << 22, 1 << 24, 51_200_000):
        f = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 1000 + rank, ess_threshold=args.ess)
        fs = torch.cuda.ExternalStream(f.state.stream, device=dev)

        def run(seed):
            f.reset(seed)
            f.step_many_device(y.data_ptr(), T, rec.data_ptr())
        for w in range(3):
            run(2000 + w)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, args.steps)
        e0.record(fs)
        for k in range(reps):
            run(3000 + k)
        e1.record(fs)
        barrier()
        t = torch.tensor([e0.elapsed_time(e1) / reps], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        res = np.frombuffer(rec.cpu().numpy().tobytes(), dtype=np.int32).reshape(T, RECORD_BYTES // 4)[:, 8]
        carry = np.zeros(T)
        carry[1:] = 1 - res[:-1]
        bytes_run = float(N) * float(np.sum(12 + 4 * carry + 12 * res))
        point = {"n_particles": N, "us_per_tick": ms / T * 1e3, "particle_steps_per_s": world * N * T / (ms / 1e3),
                 "resample_rate": float(res.mean()), "hbm_frac": bytes_run / (ms / 1e3) / 1e9 / peak}
        if rank == 0 and world == 1 and not args.no_cpu_baseline and N <= (1 << 22):
            cb = cpu_baseline(N, np.asarray(ys[:T], dtype=np.float32), args.ess, 2.0)
            point["cpu_all_cores_us_per_tick"] = cb["us_per_tick"]
        out.append(point)
        f.close()
    return {"ticks": T, "ess_threshold": args.ess, "points": out,
            "note": "device-resident CUDA-graph runs, CUDA events; hbm_frac of the measured copy peak; "
                    "cpu_all_cores_us_per_tick: the FP32 restatement of the reference tick loop on all host "
                    "cores, about 2 s of ticks from the start of the same series (N <= 2^22)"}


def bench_extensions(dev, args, lib, rank):
    """The rows beyond the plain tick, each timed on its own workload (rank 0, one GPU):
      student_t  the plain filter with Student-t state noise (nu_state=5) and observations (nu_obs=5),
                 N=2^24, the first --sweep-ticks ticks of the headline series, device-resident graph
      learning   online mu learning (K=50, rho too) on the same N=2^24 run: the host update every K ticks
                 forces tick-by-tick launches; against the same run without learning, stepped the same way
      apf        the auxiliary particle filter (two resampling stages per tick), N=2^24 and N=4096,
                 gpu_apf_step_many with host buffers
      imm        8 SV models x 4096 particles, 1000 ticks through gpu_imm_step (one host round trip per
                 tick, as the reference's API)
      step_api   gpu_bpf_step per tick on the reference suite's throughput workload (matched-DGP
                 Student-t scenario, N = 1K / 4K / 16K / 64K, 2000 ticks)
      particle_scaling  gpu_bpf_step per tick on the reference's particle-scaling benchmark
                 (N = 50K .. 1M, nu_obs 5)
      cond_resample  the reference's conditional-resampling workload (N = 300K, 3000 ticks of
                 gpu_bpf_step, always and ESS < 0.5N), beside its published RTX 5080 figures
      smc2       256 theta-particles x 512 state particles, 500 updates of gpu_bpf_smc2_update with one
                 PMMH move per outer resample; smc2_cpmmh the same with correlated-noise moves (rho 0.99)
    CUDA events on the filters' streams where the work is device-resident, else wall clock around
    synchronised calls."""
    if rank != 0:
        return None
    import numpy as np
    import torch
    import gpubpf
    from gpubpf import dgp
    out = {}
    T = args.sweep_ticks
    N = 1 << 24
    _, ys = dgp.matched_series(5000, RHO, SIG, MU, args.dgp_seed)
    y_host = np.asarray(ys[:T], dtype=np.float32)
    y = torch.tensor(y_host, device=dev)
    rec = torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev)

    def timed_device(f, seed0):
        fs = torch.cuda.ExternalStream(f.state.stream, device=dev)
        for w in range(3):
            f.reset(seed0 + w)
            f.step_many_device(y.data_ptr(), T, rec.data_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, args.steps)
        e0.record(fs)
        for k in range(reps):
            f.reset(seed0 + 10 + k)
            f.step_many_device(y.data_ptr(), T, rec.data_ptr())
        e1.record(fs)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    # Student-t state noise and observations vs Gaussian, same N and series
    g = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 7, ess_threshold=args.ess)
    ms_g = timed_device(g, 100)
    g.close()
    t = gpubpf.GpuBpf(N, RHO, SIG, MU, 5.0, 5.0, 7, ess_threshold=args.ess)
    ms_t = timed_device(t, 100)
    t.close()
    out["student_t"] = {"workload": f"N={N}, first {T} ticks, ESS<{args.ess}N, nu_state=5, nu_obs=5",
                        "us_per_tick": ms_t / T * 1e3, "particle_steps_per_s": N * T / (ms_t / 1e3),
                        "gaussian_us_per_tick": ms_g / T * 1e3, "cost_vs_gaussian": ms_t / ms_g}

    # online learning: tick-by-tick stepping with and without the score sums and updates
    Tl = min(T, 500)

    def timed_host(f, learn):
        if learn:
            f.enable_mu_learning(1, 50, 0.1, 10.0, 0.667)
            f.enable_rho_learning(True)
        f.step_many(y_host[:8].tolist())
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        f.step_many(y_host[8:8 + Tl].tolist())
        torch.cuda.synchronize(dev)
        return (time.perf_counter() - t0) * 1e3
    a = gpubpf.GpuBpf(N, RHO, SIG, 0.0, 0.0, 0.0, 7, ess_threshold=args.ess)
    ms_l = timed_host(a, True)
    mu_end = a.get_mu()
    a.close()
    b = gpubpf.GpuBpf(N, RHO, SIG, 0.0, 0.0, 0.0, 7, ess_threshold=args.ess)
    ms_nl = timed_host(b, False)
    b.close()
    out["learning"] = {"workload": f"N={N}, {Tl} ticks stepped with gpu_bpf_step_many (host buffers), mu and rho "
                                   f"learning from mu=0, K=50 (tick-by-tick launches), against the same call "
                                   f"without learning (64-tick CUDA graphs)",
                       "us_per_tick": ms_l / Tl * 1e3, "us_per_tick_without": ms_nl / Tl * 1e3,
                       "overhead": ms_l / ms_nl, "mu_after": mu_end}

    # auxiliary particle filter
    apf = {}
    y_all = np.asarray(ys, dtype=np.float32)
    for n_apf, t_apf in ((N, 300), (4096, 1000)):
        f = gpubpf.GpuApf(n_apf, RHO, SIG, MU, 0.0, 0.0, 42)
        f.step_many(y_all[:64].tolist())
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        f.step_many(y_all[64:64 + t_apf].tolist())
        torch.cuda.synchronize(dev)
        ms = (time.perf_counter() - t0) * 1e3
        f.close()
        apf[str(n_apf)] = {"ticks": t_apf, "us_per_tick": ms / t_apf * 1e3,
                           "particle_steps_per_s": n_apf * t_apf / (ms / 1e3)}
    out["apf"] = {"workload": "gpu_apf_step_many (host buffers), ticks 64.. of the headline series after 64 "
                              "warm-up ticks, two resampling stages per tick", "points": apf}

    # IMM
    grid = gpubpf.build_grid([0.95, 0.97], [0.1, 0.2], [-1.5, -1.0])
    imm = gpubpf.Imm(grid, 4096, seed=3)
    _, yi = dgp.matched_series(1064, RHO, SIG, MU, 42)
    for v in yi[:64]:
        imm.step(float(v))
    t0 = time.perf_counter()
    for v in yi[64:]:
        imm.step(float(v))
    ms = (time.perf_counter() - t0) * 1e3
    imm.close()
    out["imm"] = {"workload": f"{len(grid)} models x 4096 particles, 1000 ticks of gpu_imm_step",
                  "us_per_tick": ms, "particle_steps_per_s": len(grid) * 4096 * 1000 / (ms / 1e3)}

    # the synchronous per-tick API on the matched-DGP Student-t scenario (the reference suite's
    # throughput test, tests/test_bpf_matched_dgp.cu:560-603): 100 warm-up ticks, then 2000 ticks
    # of gpu_bpf_step, one Python call each (the reference arm times its filter in a C loop)
    ys4 = np.asarray(step_api_series(), dtype=np.float32)
    rows = {}
    for n in STEP_API_N:
        f = gpubpf.GpuBpf(n, 0.97, 0.15, -4.5, 5.0, 5.0, 42 + 900)
        for t in range(100):
            f.step(float(ys4[t % len(ys4)]))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for v in ys4.tolist():
            f.step(v)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        f.close()
        rows[str(n)] = {"us_per_tick": ms * 1e3 / len(ys4), "ticks_per_s": len(ys4) / (ms / 1e3)}
    out["step_api"] = {"workload": STEP_API_WORKLOAD, "points": rows}

    # the reference's particle-scaling benchmark, same calls
    ysc = np.asarray(scaling_series(), dtype=np.float32)
    rows = {}
    for n in SCALING_N:
        f = gpubpf.GpuBpf(n, 0.98, 0.15, -1.0, 0.0, 5.0, 42)
        for t in range(200):
            f.step(float(ysc[t]))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for v in ysc[200:].tolist():
            f.step(v)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        f.close()
        rows[str(n)] = {"us_per_tick": ms * 1e3 / (len(ysc) - 200)}
    out["particle_scaling"] = {"workload": SCALING_WORKLOAD, "points": rows}

    # the reference's conditional-resampling workload, the one per-tick figure it publishes with a
    # harness (760 ms always resampling, 448 ms with ESS < 0.5N, RTX 5080, its CUDA-C path)
    _, ycr = dgp.cond_resample_series(lambda t: 0.15)
    rows = {}
    for thr in (0.0, 0.5):
        f = gpubpf.GpuBpf(300000, 0.98, 0.15, -4.5, 0.0, 0.0, 42, ess_threshold=thr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for v in ycr.tolist():
            f.step(v)
        torch.cuda.synchronize()
        rows["always" if thr == 0.0 else "ess0.5"] = {"ms_3000_ticks": (time.perf_counter() - t0) * 1e3,
                                                       "resamples": f.state.resample_count}
        f.close()
    out["cond_resample"] = {"workload": COND_WORKLOAD, "points": rows,
                            "published_rtx5080_ms": {"always": 760.0, "ess0.5": 448.0}}

    # SMC^2, with fresh inner filters scoring the proposals and with correlated-noise (CPMMH) moves
    _, y2 = dgp.matched_series(600, RHO, SIG, MU, 11)
    for key, cp in (("smc2", 0.0), ("smc2_cpmmh", 0.99)):
        s2 = gpubpf.Smc2(256, 512, 600, seed=5)
        s2.set_moves(1, 0.5, 1.0)
        s2.set_cpmmh_rho(cp)
        for v in y2[:50]:
            s2.update(float(v))
        t0 = time.perf_counter()
        for v in y2[50:550]:
            s2.update(float(v))
        ms = (time.perf_counter() - t0) * 1e3
        mean, sd = s2.theta()
        st = s2.stats()
        s2.close()
        out[key] = {"workload": "256 theta x 512 particles, 500 updates (after 50), one PMMH move per outer "
                                "resample" + (f", correlated noise rho={cp}" if cp > 0 else ""),
                    "us_per_update": ms / 500 * 1e3, "theta_mean": [float(v) for v in mean],
                    "theta_sd": [float(v) for v in sd], "stats": st,
                    "acceptance": st["accepted"] / max(1, st["proposed"])}
    return out


def smc2_only(args):
    """The extensions' SMC^2 workload alone (256 theta x 512 particles, one PMMH move per outer
    resample, fresh inner filters): 50 warm-up updates, then args.smc2_only timed ones (wall clock
    around synchronised calls, as in the extensions)."""
    import torch
    import gpubpf
    from gpubpf import dgp
    torch.cuda.set_device(0)
    n = args.smc2_only
    _, y2 = dgp.matched_series(50 + n, RHO, SIG, MU, 11)
    s2 = gpubpf.Smc2(256, 512, 50 + n, seed=5)
    s2.set_moves(1, 0.5, 1.0)
    for v in y2[:50]:
        s2.update(float(v))
    t0 = time.perf_counter()
    for v in y2[50:]:
        s2.update(float(v))
    ms = (time.perf_counter() - t0) * 1e3
    st = s2.stats()
    s2.close()
    print(json.dumps({"workload": "SMC^2, 256 theta x 512 particles, one PMMH move per outer resample",
                      "updates": n, "us_per_update": ms / n * 1e3, "stats": st}))
    return 0


COND_WORKLOAD = ("the reference's conditional-resampling workload (tests/test_cond_resample.cu): N = 300000, "
                 "3000 ticks of gpu_bpf_step, rho 0.98, sigma_z 0.15, mu -4.5, seed 42, resampling every tick "
                 "and at ESS < 0.5N")
SCALING_N = (50000, 100000, 200000, 300000, 400000, 500000, 1000000)
SCALING_WORKLOAD = ("the reference's particle-scaling benchmark (tests/bench_particle_scaling.cu): gpu_bpf_step "
                    "per tick, rho 0.98, sigma_z 0.15, mu -1, nu_obs 5, seed 42, LCG + Box-Muller series (state "
                    "123456789), 200 warm-up then 1800 timed ticks")


def scaling_series(n=2000):
    """The series of tests/bench_particle_scaling.cu:29-38,54-63 (FP64, as there)."""
    import math
    st = 123456789

    def normal():
        nonlocal st
        st = (st * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        u1 = max((st >> 11) / float(1 << 53), 1e-15)
        st = (st * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        u2 = (st >> 11) / float(1 << 53)
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * 3.14159265358979323846 * u2)

    h, out = -1.0, []
    for _ in range(n):
        h = -1.0 + 0.98 * (h + 1.0) + 0.15 * normal()
        out.append(math.exp(h / 2.0) * normal())
    return out


STEP_API_N = (1024, 4096, 16384, 65536)
STEP_API_WORKLOAD = ("gpu_bpf_step per tick, matched-DGP Student-t scenario (rho 0.97, sigma_z 0.15, mu -4.5, "
                     "nu_state 5, nu_obs 5, DGP seed 42, 2000 ticks after 100 warm-up), filter seed 942, ESS<0.5N")


def step_api_series():
    from gpubpf import dgp
    return dgp.matched_series(2000, 0.97, 0.15, -4.5, 42, 5.0, 5.0)[1]


def bench_config1(dev, args, lib, rank):
    """Configuration 1 (the reference's CPU-runnable case): N=4096, T=1000, theta=(-1.0, 0.97, 0.15),
    resampling every tick, DGP seed 42, filter seed 42. GPU: device-resident CUDA-graph runs; CPU: the FP32
    restatement of the reference tick loop on 1 core and on all cores; total loglik vs the FP64 oracle on
    the GPU run's ancestors."""
    import numpy as np
    import torch
    import gpubpf
    from gpubpf import dgp
    from oracle import oracle
    N, T = 4096, 1000
    _, ys = dgp.matched_series(T, RHO, SIG, MU, 42)
    yh = np.asarray(ys, dtype=np.float32)
    y = torch.tensor(yh, device=dev)
    rec = torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev)
    f = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 42, ess_threshold=0.0)
    fs = torch.cuda.ExternalStream(f.state.stream, device=dev)
    for _ in range(3):
        f.reset(42)
        f.step_many_device(y.data_ptr(), T, rec.data_ptr())
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(3, args.steps)
    e0.record(fs)
    for _ in range(reps):
        f.reset(42)
        f.step_many_device(y.data_ptr(), T, rec.data_ptr())
    e1.record(fs)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    f.close()
    # log-likelihood against the FP64 oracle replaying this run's ancestors
    g = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 42, ess_threshold=0.0)
    g.record_ancestors(True)
    anc = np.zeros((T, N), dtype=np.int32)
    dll = np.zeros(T)
    for t in range(T):
        g.step(float(yh[t]))
        dll[t] = g.get_record().dloglik
        anc[t] = np.frombuffer(g.get_ancestors()[1], dtype=np.int32)
    g.close()
    o = oracle.filter_f64(N, RHO, SIG, MU, yh, seed=42, ess_threshold=0.0, anc_replay=anc,
                          flags_replay=np.ones(T, dtype=np.int32))
    err = abs(dll.sum() - o["dll"].sum()) / abs(o["dll"].sum())
    out = {"workload": "plain SV BPF, N=4096, T=1000, always resample, DGP seed 42, filter seed 42",
           "gpu": {"us_per_tick": ms / T * 1e3, "particle_steps_per_s": N * T / (ms / 1e3)},
           "loglik": float(dll.sum()), "loglik_oracle_fp64": float(o["dll"].sum()), "loglik_rel_err": err}
    if rank == 0 and not args.no_cpu_baseline:
        cpu = {}
        for label, nt in (("1_core", 1), ("all_cores", os.cpu_count() or 1)):
            oracle.lib(True)
            t0 = time.perf_counter()
            oracle.ref_run(N, RHO, SIG, MU, yh, seed=42, ess_threshold=0.0, nthreads=nt, native=True)
            dt = time.perf_counter() - t0
            cpu[label] = {"cores": nt, "us_per_tick": dt / T * 1e6, "particle_steps_per_s": N * T / dt}
        out["cpu_reference_restatement"] = cpu
    return out


def bench_gradient(dev, args, lib, rank, world, barrier):
    """Configuration 3: theta=(mu=-0.8, phi=0.95, sigma_eta=0.25), N=2^20, T=2000, DGP seed 42 with the same
    theta, resampling every tick. Times the plain forward (device graph), the taped forward and the adjoint
    backward (each one CUDA graph) with events on their streams; checks the adjoint at full size against the
    FP64 replay's forward-mode tangents and the 5-point central difference (step 1e-3*|theta_k|) of the FP64
    replay under common random numbers with the taped ancestors. Multi-GPU: replicas (seed per rank)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import gpubpf
    from gpubpf import dgp
    mu, rho, sig = -0.8, 0.95, 0.25
    N, T, seed = args.grad_n, args.grad_ticks, 42 + rank
    _, ys = dgp.matched_series(T, rho, sig, mu, 42)
    y = torch.tensor(np.asarray(ys, dtype=np.float32), device=dev)
    reps = max(1, args.steps)

    def timed(stream, fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        barrier()
        t = torch.tensor([e0.elapsed_time(e1) / reps], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # plain forward (the drop-in path), always resample
    f = gpubpf.GpuBpf(N, rho, sig, mu, 0.0, 0.0, seed, ess_threshold=0.0)
    rec = torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev)
    fs = torch.cuda.ExternalStream(f.state.stream, device=dev)

    def plain():
        f.reset(seed)
        f.step_many_device(y.data_ptr(), T, rec.data_ptr())
    for _ in range(3):
        plain()
    barrier()
    ms_plain = timed(fs, plain)
    f.close()

    tape = gpubpf.GradTape(N, T)
    ts = tape.stream
    for _ in range(3):
        tape.forward((mu, rho, sig), y, seed=seed)
        tape.backward()
    barrier()
    ms_fwd = timed(ts, lambda: tape.forward((mu, rho, sig), y, seed=seed))
    ms_bwd = timed(ts, tape.backward)
    ms_both = timed(ts, lambda: (tape.forward((mu, rho, sig), y, seed=seed), tape.backward()))
    ll = float(tape.forward((mu, rho, sig), y, seed=seed).item())
    g = tape.backward().cpu().numpy()
    rep = tape.replay((mu, rho, sig)).cpu().numpy()
    fd5 = tape.fd_gradient((mu, rho, sig), rel=1e-3, points=5)
    fd3 = tape.fd_gradient((mu, rho, sig), rel=1e-3, points=3)
    scale = float(np.max(np.abs(g)))
    out = {
        "workload": f"SV gradient, theta=(mu={mu}, phi={rho}, sigma_eta={sig}), N={N}, T={T}, always resample, "
                    f"DGP seed 42",
        "ms_forward_plain": ms_plain, "ms_forward_taped": ms_fwd, "ms_backward": ms_bwd,
        "ms_forward_plus_backward": ms_both,
        "grad_over_forward": ms_both / ms_plain,
        "us_per_tick": {"plain_forward": ms_plain / T * 1e3, "taped_forward": ms_fwd / T * 1e3,
                        "backward": ms_bwd / T * 1e3},
        "loglik": ll, "grad": g.tolist(),
        "replay_fp64": {"loglik": float(rep[0]), "grad": rep[1:].tolist(),
                        "rel_err": float(np.max(np.abs(g - rep[1:])) / scale)},
        "fd_5point": {"grad": fd5.tolist(), "rel_err": float(np.max(np.abs(g - fd5)) / scale),
                      "step": "1e-3*|theta_k|"},
        "fd_3point": {"grad": fd3.tolist(), "rel_err": float(np.max(np.abs(g - fd3)) / scale)},
        "tape_bytes": gpubpf.GradTape.tape_bytes(N, T), "checkpoint_every": tape.checkpoint_every,
        "timing": "CUDA events on the filter / tape stream, mean of --steps runs after 3 warm-ups, max over ranks",
    }
    tape.close()
    return out


def bench_batch_gradient(dev, args, lib, rank, world, barrier):
    """Configuration 5: B=256 filters with N=8192, theta drawn as in configuration 4, T=4000 ticks of the
    regime-switching series (mu alternating -1.5 / 0.0 every 500 ticks, phi=0.97, sigma_eta=0.2, seed 42);
    one iteration = forward + backward of every filter (per-filter loglik and d loglik / d theta). Timed
    against the batched forward alone on the same filters; two filters are checked against plain gradient
    tapes. Filters are sharded across ranks by LPT on N."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import gpubpf
    from gpubpf import configs, dgp, parallel
    B, T = args.bgrad_filters, args.bgrad_ticks
    allf = configs.config5(B)
    _, fl = parallel.shard(allf, rank, world)
    _, ys = dgp.regime_series(T, seed=42)
    y = np.asarray(ys, dtype=np.float32)
    y_d = torch.tensor(y, device=dev)
    b = gpubpf.GpuBpfBatch(fl, ess_threshold=0.0)
    bs = torch.cuda.ExternalStream(b.stream, device=dev)
    ll = torch.zeros(len(fl), dtype=torch.float64, device=dev)
    g = torch.zeros(3 * len(fl), dtype=torch.float64, device=dev)
    reps = max(1, args.steps)

    def timed(fn):
        for _ in range(2):
            fn()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bs)
        for _ in range(reps):
            fn()
        e1.record(bs)
        barrier()
        t = torch.tensor([e0.elapsed_time(e1) / reps], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms_fwd = timed(lambda: b.run_device(y_d.data_ptr(), T, ll.data_ptr()))
    ms_both = timed(lambda: b.grad_run(y_d.data_ptr(), T, ll.data_ptr(), g.data_ptr()))
    llv = ll.cpu().numpy()
    gv = g.cpu().numpy().reshape(-1, 3)
    tape_bytes = b.grad_tape_bytes(T)
    b.close()
    errs = []
    for i in (0, len(fl) - 1):
        f = fl[i]
        tape = gpubpf.GradTape(f["n_particles"], T, checkpoint_every=8)
        tape.forward((f["mu"], f["rho"], f["sigma_z"]), y_d, seed=f["seed"])
        pg = tape.backward().cpu().numpy()
        tape.close()
        errs.append(float(np.max(np.abs(gv[i] - pg)) / np.max(np.abs(pg))))
    steps = float(sum(f["n_particles"] for f in allf)) * T
    return {"workload": f"batched gradient, B={B} filters x N=8192, T={T} regime-switching series "
                        f"(mu -1.5/0.0 every 500 ticks, phi=0.97, sigma_eta=0.2, seed 42), always resample",
            "ms_per_iteration": ms_both, "ms_forward_only": ms_fwd, "grad_over_forward": ms_both / ms_fwd,
            "particle_steps_per_s": steps / (ms_both / 1e3), "unit": "particle-steps/s (forward+backward)",
            "loglik_finite": bool(np.all(np.isfinite(llv))), "grad_finite": bool(np.all(np.isfinite(gv))),
            "check_vs_plain_tape_rel_err": errs, "tape_bytes": tape_bytes,
            "shard": f"LPT on N over {world} rank(s)"}


def headline_config(args, world):
    """The `config` of the headline line, identical in both arms (same workload, same keys)."""
    return {"workload": f"plain SV BPF, N={args.n}, T={args.ticks}, ESS<{args.ess}N, theta=(mu={MU}, phi={RHO}, "
                        f"sigma_eta={SIG}), DGP seed {args.dgp_seed}",
            "n_particles": args.n, "ticks": args.ticks, "ess_threshold": args.ess, "l2": L2_NOTE,
            "parallelism": f"replicas x{world}" if world > 1 else "single filter"}


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def spawn_ranks(n):
    """`bench.py --gpus N` started without a launcher: start N ranks of this same command line (one
    process per GPU) through torch.distributed.run on 127.0.0.1 and return its exit status. Rank 0
    prints the JSON line."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def plumbing_check(args):
    """The multi-rank path of this bench without a GPU (gloo): every rank takes its LPT shard of the
    configuration-4 filters, produces one stand-in value per filter (a function of the filter alone),
    the values are gathered with gpubpf.parallel.gather_results and a per-rank time is max-reduced,
    as the GPU path does. Rank 0 prints one JSON line saying whether every filter came back once and
    unchanged."""
    import datetime
    import torch
    import torch.distributed as dist
    from gpubpf import configs, parallel
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    allf = configs.config4(args.batch_filters)

    def stand_in(f):
        return f["n_particles"] * 1e-3 + f["mu"] + 10.0 * f["rho"] + 100.0 * f["sigma_z"] + f["seed"] * 1e-6

    idx, mine = parallel.shard(allf, rank, world)
    vals = [stand_in(f) for f in mine]
    full = parallel.gather_results(idx, vals, len(allf)) if world > 1 else vals
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        ok = len(full) == len(allf) and all(a == stand_in(f) for a, f in zip(full, allf))
        print(json.dumps({"plumbing_check": True, "n_ranks": world, "filters": len(allf), "gathered_ok": ok,
                          "max_over_ranks": float(t.item()), "shard_sizes": [len(p) for p in parallel.lpt_partition(
                              [f["n_particles"] for f in allf], world)]}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def headline_parity(N, y, ess, ticks, seed=42):
    """The headline workload's first `ticks` ticks followed by the FP64 oracle in lock step: the
    device filter runs tick by tick through the C ABI with its ancestors recorded, the oracle
    replays each tick's resampling decision and ancestors, and each resampling tick's ancestors are
    recomputed by the oracle's fixed-point mirror from the device's weights. Checker only: nothing
    here is timed."""
    import numpy as np
    import gpubpf
    from oracle import oracle
    f = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, seed, ess_threshold=ess)
    f.record_ancestors(True)
    o = oracle.F64Filter(N, RHO, SIG, MU, seed=seed, ess_threshold=ess)
    gd, od, n_res, n_exact = [], [], 0, 0
    try:
        for t in range(ticks):
            f.step(float(y[t]))
            r = f.get_record()
            anc = None
            if r.resampled:
                anc = np.frombuffer(f.get_ancestors()[1], dtype=np.int32)
                w, te, u23 = f.get_resample_inputs()
                ref = oracle.resample_fixed(np.frombuffer(w, dtype=np.float32), np.frombuffer(te, dtype=np.int32), u23)
                n_res += 1
                n_exact += int(np.array_equal(anc, ref))
            q = o.tick(y[t], anc=anc, flag=int(r.resampled))
            gd.append(r.dloglik)
            od.append(q["dll"])
    finally:
        f.close()
        o.close()
    gd, od = np.asarray(gd), np.asarray(od)
    return {"n_particles": N, "ticks": ticks, "filter_seed": seed,
            "loglik": float(gd.sum()), "loglik_oracle_fp64": float(od.sum()),
            "loglik_rel_err": float(abs(gd.sum() - od.sum()) / abs(od.sum())),
            "max_abs_increment_err": float(np.max(np.abs(gd - od))),
            "resampling_ticks": n_res, "ancestors_bit_exact_ticks": n_exact,
            "method": "FP64 oracle (oracle/bpf_oracle.c orc_f64_tick) in lock step on the device's ancestors; "
                      "ancestors vs orc_resample_fixed on the device's weights"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    from gpubpf import dgp
    _, ys = dgp.matched_series(args.ticks, RHO, SIG, MU, args.dgp_seed)
    y = np.asarray(ys, dtype=np.float32)
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(args.n, y, args.ess, per_step)
    vals, uspt = [], []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_baseline(args.n, y, args.ess, per_step)
        vals.append(r["value"]); uspt.append(r["us_per_tick"])
    wall = time.perf_counter() - t0
    value = statistics.mean(vals)
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / max(1, args.steps) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": headline_config(args, int(os.environ.get("WORLD_SIZE", "1"))),
        "us_per_tick": statistics.mean(uspt),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": r["cores"], "kind": "port",
                         "sample": r["sample"]},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu(args, y),
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu(args, y):
    """The reference's own GPU filter (its PTX edition, built into oracle/_ref/ from the reference
    sources) on this GPU, same workload: a fresh gpu_bpf_create per step (untimed), then the T-tick
    gpu_bpf_step_async loop with its per-tick host ESS decision, wall-clocked to the final stream
    synchronise. Also configuration 1 (N=4096, T=1000, always resample). None when the library
    was not built or no GPU is visible."""
    try:
        import torch
        from oracle import refgpu
        if not (refgpu.available() and torch.cuda.is_available()):
            return None
    except Exception:
        return None
    import numpy as np

    def timed(n, yy, ess, steps, warmup):
        ms, last, count = [], None, 0
        for k in range(warmup + steps):
            f = refgpu.RefGpuFilter(n, RHO, SIG, MU, seed=42, ess_threshold=ess)
            t, hm, ll = f.time_run(yy)
            count = f.resample_count
            f.close()
            if k >= warmup:
                ms.append(t)
                last = (hm, ll)
        m = statistics.mean(ms)
        return {"value": n * len(yy) / (m / 1e3), "unit": "particle-steps/s", "ms_per_step": m,
                "us_per_tick": m * 1e3 / len(yy), "resample_count": count,
                "last_tick": {"h_mean": last[0], "log_lik": last[1]}}

    out = timed(args.n, y, args.ess, max(1, min(args.steps, 3)), 1)
    out["kind"] = ("reference PTX edition (gpu_bpf/gpu_bpf_ptx_full.cu + ptx_assembly/bpf_kernels_full.ptx, "
                   "JIT for sm_100a) on this GPU")
    out["workload"] = f"N={args.n}, T={len(y)}, ESS<{args.ess}N, DGP seed {args.dgp_seed}, filter seed 42"
    from gpubpf import dgp
    _, y1 = dgp.matched_series(1000, RHO, SIG, MU, 42)
    c1 = timed(4096, np.asarray(y1, dtype=np.float32), 0.0, 3, 1)
    out["config1"] = {"us_per_tick": c1["us_per_tick"], "value": c1["value"], "unit": c1["unit"],
                      "workload": "N=4096, T=1000, always resample, DGP seed 42"}
    # the reference's auxiliary particle filter (gpu_apf_step), same points as the extensions section
    _, ya = dgp.matched_series(1064, RHO, SIG, MU, args.dgp_seed)
    ya = np.asarray(ya, dtype=np.float32)
    out["apf"] = {str(n): {"ticks": t, "us_per_tick": refgpu.apf_time(n, RHO, SIG, MU, ya[:64 + t]) * 1e3}
                  for n, t in ((args.n, 300), (4096, 1000))}
    # its synchronous per-tick API on the suite's throughput workload (same points as the extensions)
    ys4 = np.asarray(step_api_series(), dtype=np.float32)
    rows = {}
    for n in STEP_API_N:
        f = refgpu.RefGpuFilter(n, 0.97, 0.15, -4.5, 5.0, 5.0, seed=42 + 900)
        ms = f.time_steps(ys4, warmup=100)
        f.close()
        rows[str(n)] = {"us_per_tick": ms * 1e3 / len(ys4), "ticks_per_s": len(ys4) / (ms / 1e3)}
    out["step_api"] = {"workload": STEP_API_WORKLOAD + "; gpu_bpf_step in a C loop", "points": rows}
    ysc = np.asarray(scaling_series(), dtype=np.float32)
    rows = {}
    for n in SCALING_N:
        f = refgpu.RefGpuFilter(n, 0.98, 0.15, -1.0, 0.0, 5.0, seed=42)
        f.run(ysc[:200])                                  # warm-up ticks, as the benchmark's
        ms = f.time_steps(ysc[200:], warmup=0)
        f.close()
        rows[str(n)] = {"us_per_tick": ms * 1e3 / (len(ysc) - 200)}
    out["particle_scaling"] = {"workload": SCALING_WORKLOAD + "; gpu_bpf_step in a C loop", "points": rows}
    _, ycr = dgp.cond_resample_series(lambda t: 0.15)
    rows = {}
    for thr in (0.0, 0.5):
        f = refgpu.RefGpuFilter(300000, 0.98, 0.15, -4.5, seed=42, ess_threshold=thr)
        rows["always" if thr == 0.0 else "ess0.5"] = {"ms_3000_ticks": f.time_steps(ycr, warmup=0),
                                                       "resamples": f.resample_count}
        f.close()
    out["cond_resample"] = {"workload": COND_WORKLOAD + "; gpu_bpf_step in a C loop", "points": rows}
    return out


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    if args.plumbing_check:
        return plumbing_check(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.smc2_only:
        return smc2_only(args)

    import numpy as np
    import torch
    import torch.distributed as dist
    import gpubpf
    from gpubpf import dgp

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=dev)

    lib = gpubpf.load()
    N, T = args.n, args.ticks
    _, ys = dgp.matched_series(T, RHO, SIG, MU, args.dgp_seed)
    y_host = np.asarray(ys, dtype=np.float32)
    y_dev = torch.from_numpy(y_host).to(dev)
    rec_dev = torch.zeros(T * RECORD_BYTES, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    f = gpubpf.GpuBpf(N, RHO, SIG, MU, 0.0, 0.0, 1000 + rank, ess_threshold=args.ess)
    ext = torch.cuda.ExternalStream(f.state.stream, device=dev)

    def one_run(seed):
        f.reset(seed)
        f.step_many_device(y_dev.data_ptr(), T, rec_dev.data_ptr())
        with torch.cuda.stream(ext):
            flush.zero_()

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    # ---------------- device-resident timed region -------------------------
    for w in range(max(3, args.warmup)):
        one_run(2000 + w)
    barrier()
    props = torch.cuda.get_device_properties(dev)
    gpu_id = str(getattr(props, "uuid", "") or "")
    if gpu_id and not gpu_id.startswith("GPU-"):
        gpu_id = "GPU-" + gpu_id
    clk = ClockSampler(gpu_id or str(local))
    launches0 = lib.gpu_bpf_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for k in range(args.steps):
        one_run(3000 + k)
    e1.record(ext)
    barrier()
    clocks = clk.stop()
    launches = lib.gpu_bpf_launch_count() - launches0
    ms = e0.elapsed_time(e1)
    t_max = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    value = world * N * T * args.steps / (ms_max / 1e3)

    recs = rec_dev.cpu().numpy().view(np.uint8)
    resampled = np.frombuffer(recs.tobytes(), dtype=np.int32).reshape(T, RECORD_BYTES // 4)[:, 8]
    resample_rate = float(resampled.mean())

    # ---------------- per-kernel durations (profiled pass) -----------------
    f.profile(True)
    f.reset(3000)
    f.step_many_device(y_dev.data_ptr(), T, rec_dev.data_ptr())
    p1_ms, plan_ms, p2_ms, n1 = f.profile_read()
    n2 = n1
    f.profile(False)
    rec = np.frombuffer(rec_dev.cpu().numpy().tobytes(), dtype=np.int32).reshape(T, RECORD_BYTES // 4)[:, 8]
    carry = np.zeros(T, dtype=np.int64)
    carry[1:] = 1 - rec[:-1]
    bytes_p1 = float(N) * float(np.sum(12 + 4 * carry))
    bytes_p2 = float(N) * 12.0 * float(rec.sum())
    peak, peak_kind = load_peaks()
    traffic = load_traffic()
    ach1 = bytes_p1 / (p1_ms / 1e3) / 1e9
    ach2 = bytes_p2 / (p2_ms / 1e3) / 1e9 if p2_ms > 0 else 0.0
    dominant = "pass1" if p1_ms >= p2_ms else "pass2"
    ach, nl, tms = (ach1, n1, p1_ms) if dominant == "pass1" else (ach2, n2, p2_ms)
    tr = traffic.get(dominant + "_kernel")
    roofline = {
        "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
        "traffic": (tr * N if tr is not None else None),
        "kernel": dominant + "_kernel", "peak_source": peak_kind,
        "algorithmic_bytes_per_launch": (bytes_p1 if dominant == "pass1" else bytes_p2) / max(1, nl),
        "avg_launch_us": tms / max(1, nl) * 1e3,
        "pass1": {"ms": p1_ms, "launches": n1, "GBps": ach1, "frac": ach1 / peak},
        "pass2": {"ms": p2_ms, "launches": n2, "GBps": ach2, "frac": ach2 / peak},
        "plan": {"ms": plan_ms, "launches": n1, "us_per_launch": plan_ms / max(1, n1) * 1e3},
        "tick": {"GBps": (bytes_p1 + bytes_p2) / ((p1_ms + plan_ms + p2_ms) / 1e3) / 1e9,
                 "frac": (bytes_p1 + bytes_p2) / ((p1_ms + plan_ms + p2_ms) / 1e3) / 1e9 / peak},
        "bytes_model": "pass1 12 B/particle (+4 carried weight on ticks after a skipped resample); "
                       "pass2 12 B/particle on resampling ticks",
    }

    # ---------------- end-to-end through the host-buffer C ABI -------------
    e2e = None
    if not args.no_e2e:
        out_res = None
        for w in range(2):
            f.reset(4000 + w)
            f.step_many(y_host.tolist())
        barrier()
        import ctypes as C
        ya = (C.c_float * T)(*y_host.tolist())
        outa = (gpubpf.BpfResult * T)()
        reca = (gpubpf.BpfTickRecord * T)()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e2.record(ext)
        for k in range(args.steps):
            f.reset(5000 + k)
            gpubpf._lib.check(lib.gpu_bpf_step_many(f._s, ya, T, outa, reca), "gpu_bpf_step_many")
        e3.record(ext)
        barrier()
        wall = time.perf_counter() - t0
        ms_e2e = max(e2.elapsed_time(e3), wall * 1e3)
        t2 = torch.tensor([ms_e2e], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        e2e = {"value": world * N * T * args.steps / (float(t2.item()) / 1e3), "unit": "particle-steps/s",
               "h2d_bytes_per_step": 4 * T,
               "d2h_bytes_per_step": RECORD_BYTES * T + DEVSTATE_BYTES,
               "api": "gpu_bpf_reset + gpu_bpf_step_many(host y[T], host BpfResult[T], host BpfTickRecord[T])"}

    f.close()
    sweep = None if args.no_sweep else bench_sweep(dev, args, lib, rank, world, barrier)
    config1 = None if args.no_config1 else bench_config1(dev, args, lib, rank)
    batched = None if args.no_batched else bench_batched(dev, args, lib, rank, world, barrier)
    gradient = None if args.no_gradient else bench_gradient(dev, args, lib, rank, world, barrier)
    batch_gradient = None if args.no_batch_gradient else bench_batch_gradient(dev, args, lib, rank, world, barrier)
    extensions = None if (args.no_extensions or world > 1) else bench_extensions(dev, args, lib, rank)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(N, y_host, args.ess, args.cpu_seconds)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if args.parity_ticks > 0:
            parity = headline_parity(N, y_host, args.ess, min(args.parity_ticks, T))

    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (reference matched DGP, seed 7)",
            "config": headline_config(args, world),
            "us_per_tick": ms_max / (args.steps * T) * 1e3,
            "resample_rate": resample_rate,
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": e2e,
            "clocks": clocks,
            "sweep": sweep,
            "config1": config1,
            "batched": batched,
            "gradient": gradient,
            "batch_gradient": batch_gradient,
            "extensions": extensions,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
