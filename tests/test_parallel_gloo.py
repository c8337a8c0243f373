"""CPU tests of the multi-GPU placement logic: LPT partition and the gather of
per-filter results across ranks, run as two gloo processes (world_size 2).
The per-filter values come from the CPU oracle on tiny filters, so the test
needs no GPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG_DIR, REPO


def test_lpt_partition_balanced_and_deterministic():
    import sys
    sys.path.insert(0, PKG_DIR)
    from gpubpf import configs, parallel
    fl = configs.config4(1024)
    costs = [f["n_particles"] for f in fl]
    for world in (1, 2, 4, 8):
        parts = parallel.lpt_partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(1024))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)          # LPT bound
        assert parts == parallel.lpt_partition(costs, world)  # same on every rank


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_q):
    import sys
    sys.path.insert(0, REPO)
    sys.path.insert(0, PKG_DIR)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from gpubpf import configs, dgp, parallel
    from oracle import oracle
    fl = [dict(f, n_particles=64 + 13 * i) for i, f in enumerate(configs.batch_thetas(10))]
    _, ys = dgp.matched_series(30, 0.97, 0.2, -1.0, 42)
    y = np.asarray(ys, dtype=np.float32)
    idx, mine = parallel.shard(fl, rank, world)
    vals = [oracle.filter_f64(f["n_particles"], f["rho"], f["sigma_z"], f["mu"], y, seed=f["seed"])["dll"].sum()
            for f in mine]
    full = parallel.gather_results(idx, vals, len(fl))
    if rank == 0:
        result_q.put(full)
    dist.destroy_process_group()


def test_sharded_batch_gathers_every_filter():
    import sys
    sys.path.insert(0, REPO)
    sys.path.insert(0, PKG_DIR)
    from gpubpf import configs, dgp
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fl = [dict(f, n_particles=64 + 13 * i) for i, f in enumerate(configs.batch_thetas(10))]
    _, ys = dgp.matched_series(30, 0.97, 0.2, -1.0, 42)
    y = np.asarray(ys, dtype=np.float32)
    ref = [oracle.filter_f64(f["n_particles"], f["rho"], f["sigma_z"], f["mu"], y, seed=f["seed"])["dll"].sum()
           for f in fl]
    np.testing.assert_allclose(full, ref, rtol=0, atol=0)


def test_bench_spawns_ranks_and_gathers():
    """`bench.py --gpus 2` started without a launcher starts its own two ranks (torch.distributed.run
    on 127.0.0.1); with --plumbing-check they run on CPU over gloo: LPT shards of the
    configuration-4 filters, the gather of per-filter values and the max over ranks, as the GPU
    path does."""
    import json
    import subprocess
    import sys
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env.pop("RANK", None)
    env.pop("LOCAL_RANK", None)
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--plumbing-check"],
                         cwd=REPO, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["n_ranks"] == 2 and d["filters"] == 1024 and d["gathered_ok"]
    assert d["max_over_ranks"] == 2.0 and sum(d["shard_sizes"]) == 1024
