#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference checkout is readable ($BPF_REFERENCE, else a directory
named `reference` beside this repository). Nothing at test time reads the
reference; only the JSON files written here are committed.

Fixtures
  rng_diag_seed42.json   the known-answer block of tests/test_rng_diag.cu:76-96
                         (PCG32 state after bpf_init_rng and first output, seed 42,
                         particles 0-7), compiled with gcc from the reference
                         lines and run here
  host_u_stream.json     host_pcg32 / host_pcg32_float of
                         gpu_bpf/gpu_bpf_ptx_full.cu:241-251 from the state
                         seed*67890+12345 (:353), compiled from the reference lines
  dgp_series.json        generate_matched_series of tests/test_bpf_matched_dgp.cu
                         (:59-99 helpers, :105-127 data struct, :141-175) for the
                         benchmark inputs, compiled from the reference lines
  dgp_scenarios.json     the nine matched-DGP scenarios of tests/test_bpf_matched_dgp.cu:181-285
                         (parameters parsed from the gen_* functions) and, for each, the
                         head and sums of generate_matched_series with Student-t noises
                         (:88-99) at the suite's seeds (base 42 + scenario index, T = 5000),
                         compiled from the reference lines
  systematic_resample.json  tests/diff_bpf.py:35-56 systematic_resample run on
                         seeded log-weights (imports the reference module)

The reference source lines are copied only into a temporary directory for
compilation; they are never written into this repository.
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import re
import struct
import subprocess
import sys
import tempfile

# The reference tree: $BPF_REFERENCE, else a checkout named `reference` beside this repository.
REF = os.environ.get("BPF_REFERENCE") or os.path.join(os.path.dirname(os.path.abspath(__file__)), os.pardir,
                                                      os.pardir, os.pardir, "reference")
OUT = os.path.dirname(os.path.abspath(__file__))


def ref_lines(rel: str, a: int, b: int) -> str:
    with open(os.path.join(REF, rel), encoding="utf-8", errors="replace") as f:
        lines = f.read().splitlines()
    return "\n".join(lines[a - 1:b]) + "\n"


def compile_run(src: str, tmp: str, name: str) -> str:
    c = os.path.join(tmp, name + ".c")
    exe = os.path.join(tmp, name)
    with open(c, "w") as f:
        f.write(src)
    subprocess.run(["gcc", "-O0", "-std=gnu11", c, "-o", exe, "-lm"], check=True)
    return subprocess.run([exe], check=True, capture_output=True, text=True).stdout


def rng_diag(tmp: str) -> dict:
    body = ref_lines("tests/test_rng_diag.cu", 76, 96)
    src = "#include <stdio.h>\nint main(void) {\n" + body + "\nreturn 0;\n}\n"
    out = compile_run(src, tmp, "rng_diag")
    rows = []
    for m in re.finditer(r"particle (\d+): expected_state=([0-9a-f]+)\s+pcg_out=([0-9a-f]+)\s+u=([0-9.]+)", out):
        rows.append({"particle": int(m.group(1)), "state": m.group(2), "pcg_out": m.group(3),
                     "u": float(m.group(4))})
    assert len(rows) == 8, out
    return {"source": "tests/test_rng_diag.cu:76-96 (compiled and run)", "seed": 42, "rows": rows}


def host_u(tmp: str) -> dict:
    funcs = ref_lines("gpu_bpf/gpu_bpf_ptx_full.cu", 241, 251)
    seed_expr = ref_lines("gpu_bpf/gpu_bpf_ptx_full.cu", 353, 353)
    assert "67890ULL" in seed_expr and "12345ULL" in seed_expr, seed_expr
    drv = r"""
#include <stdio.h>
%s
int main(void) {
  int seeds[3] = {42, 7, -3};
  for (int k = 0; k < 3; ++k) {
    int seed = seeds[k];
    unsigned long long st = (unsigned long long)seed * 67890ULL + 12345ULL;
    printf("seed %%d", seed);
    for (int i = 0; i < 16; ++i) printf(" %%u", host_pcg32(&st));
    printf("\n");
    st = (unsigned long long)seed * 67890ULL + 12345ULL;
    printf("useed %%d", seed);
    for (int i = 0; i < 16; ++i) { float u = host_pcg32_float(&st); unsigned b; memcpy(&b, &u, 4); printf(" %%08x", b); }
    printf("\n");
  }
  return 0;
}
""" % funcs
    drv = "#include <string.h>\n" + drv
    out = compile_run(drv, tmp, "host_u")
    res = {"source": "gpu_bpf/gpu_bpf_ptx_full.cu:241-251,353 (compiled and run)", "streams": {}}
    for line in out.splitlines():
        parts = line.split()
        if parts[0] == "seed":
            res["streams"].setdefault(parts[1], {})["u32"] = [int(v) for v in parts[2:]]
        elif parts[0] == "useed":
            res["streams"].setdefault(parts[1], {})["float_bits"] = parts[2:]
    return res


def dgp(tmp: str) -> dict:
    rel = "tests/test_bpf_matched_dgp.cu"
    helpers = ref_lines(rel, 59, 99)
    data = ref_lines(rel, 105, 127)
    free_ = ref_lines(rel, 129, 135)
    gen = ref_lines(rel, 141, 175)
    cases = [
        # (label, seed, rho, sigma_z, mu, T) -- the benchmark configurations
        ("config1_seed42", 42, 0.97, 0.15, -1.0, 1000),
        ("config2_seed7", 7, 0.97, 0.15, -1.0, 5000),
        ("config3_seed42", 42, 0.95, 0.25, -0.8, 2000),
        ("config4_seed42", 42, 0.97, 0.2, -1.0, 2000),
    ]
    drv = ["#include <stdio.h>", "#include <stdlib.h>", "#include <stdint.h>", "#include <math.h>",
           helpers, data, free_, gen, "int main(void) {"]
    for label, seed, rho, sig, mu, T in cases:
        drv.append(f'  {{ pcg32_dgp_t rng; pcg32_dgp_seed(&rng, {seed}ULL);'
                   f' MatchedTestData* d = alloc_matched_data({T});'
                   f' generate_matched_series(d, {rho}, {sig}, {mu}, 0.0, 0.0, &rng);'
                   f' printf("case {label}\\n");'
                   f' for (int t = 0; t < {T}; ++t) printf("%.17g %.17g\\n", d->true_h[t], d->returns[t]);'
                   f' free_matched_data(d); }}')
    drv.append("  return 0;\n}\n")
    out = compile_run("\n".join(drv), tmp, "dgp")
    res = {"source": f"{rel}:59-99,105-135,141-175 (compiled and run), nu_state = nu_obs = 0", "cases": {}}
    cur = None
    series = {}
    for line in out.splitlines():
        if line.startswith("case "):
            cur = line.split()[1]
            series[cur] = ([], [])
        else:
            h, y = line.split()
            series[cur][0].append(float(h))
            series[cur][1].append(float(y))
    for label, seed, rho, sig, mu, T in cases:
        hs, ys = series[label]
        blob = struct.pack(f"<{2 * T}d", *hs, *ys)
        keep = T if T <= 1000 else 300
        res["cases"][label] = {
            "seed": seed, "rho": rho, "sigma_z": sig, "mu": mu, "T": T,
            "sha256_h_then_y_f64le": hashlib.sha256(blob).hexdigest(),
            "true_h_head": hs[:keep], "y_head": ys[:keep],
            "sum_h": sum(hs), "sum_y2": sum(v * v for v in ys),
        }
    return res


def dgp_scenarios(tmp: str) -> dict:
    rel = "tests/test_bpf_matched_dgp.cu"
    src = ref_lines(rel, 181, 285)
    pat = re.compile(r'scenario_id\s*=\s*(\d+);\s*d->scenario_name\s*=\s*"([^"]+)";.*?'
                     r'generate_matched_series\(d,\s*([-0-9.]+),\s*([-0-9.]+),\s*([-0-9.]+),\s*([-0-9.]+),'
                     r'\s*([-0-9.]+),\s*&rng\)', re.S)
    scen = [(int(m.group(1)), m.group(2), *(float(m.group(k)) for k in range(3, 8))) for m in pat.finditer(src)]
    assert len(scen) == 9, scen
    helpers = ref_lines(rel, 59, 99)
    data = ref_lines(rel, 105, 127)
    free_ = ref_lines(rel, 129, 135)
    gen = ref_lines(rel, 141, 175)
    T, base_seed = 5000, 42                      # the suite's defaults (:739-742)
    drv = ["#include <stdio.h>", "#include <stdlib.h>", "#include <stdint.h>", "#include <math.h>",
           helpers, data, free_, gen, "int main(void) {"]
    for i, (sid, name, rho, sig, mu, nus, nuo) in enumerate(scen):
        drv.append(f'  {{ pcg32_dgp_t rng; pcg32_dgp_seed(&rng, {base_seed + i}ULL);'
                   f' MatchedTestData* d = alloc_matched_data({T});'
                   f' generate_matched_series(d, {rho!r}, {sig!r}, {mu!r}, {nus!r}, {nuo!r}, &rng);'
                   f' printf("case {sid}\\n");'
                   f' for (int t = 0; t < {T}; ++t) printf("%.17g %.17g\\n", d->true_h[t], d->returns[t]);'
                   f' free_matched_data(d); }}')
    drv.append("  return 0;\n}\n")
    out = compile_run("\n".join(drv), tmp, "dgp_scen")
    series, cur = {}, None
    for line in out.splitlines():
        if line.startswith("case "):
            cur = int(line.split()[1])
            series[cur] = ([], [])
        else:
            h, y = line.split()
            series[cur][0].append(float(h))
            series[cur][1].append(float(y))
    res = {"source": f"{rel}:59-99,105-135,141-175,181-285 (parsed, compiled and run); suite defaults T = 5000, "
                     f"base seed 42, scenario i (0-based) generated with seed 42 + i (:462-464)",
           "T": T, "base_seed": base_seed, "scenarios": []}
    for i, (sid, name, rho, sig, mu, nus, nuo) in enumerate(scen):
        hs, ys = series[sid]
        res["scenarios"].append({
            "id": sid, "name": name, "seed": base_seed + i, "rho": rho, "sigma_z": sig, "mu": mu,
            "nu_state": nus, "nu_obs": nuo, "true_h_head": hs[:300], "y_head": ys[:300],
            "sum_h": sum(hs), "sum_y2": sum(v * v for v in ys)})
    return res


def systematic() -> dict:
    import torch
    spec = importlib.util.spec_from_file_location("ref_diff_bpf", os.path.join(REF, "tests", "diff_bpf.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    cases = []
    for n, seed in ((16, 1), (64, 2), (1000, 3), (4096, 4)):
        g = torch.Generator().manual_seed(1000 + seed)
        log_w = (torch.randn(n, generator=g) * 2.0).to(torch.float32)
        torch.manual_seed(seed)
        u_probe = torch.rand(1).item() / n        # the u systematic_resample will draw
        torch.manual_seed(seed)
        idx, _ = mod.systematic_resample(log_w)
        cases.append({
            "n": n,
            "log_w_f32le_hex": struct.pack(f"<{n}f", *log_w.tolist()).hex(),
            "u_over_n": u_probe,
            "indices": idx.tolist(),
        })
    return {"source": "tests/diff_bpf.py:35-56 systematic_resample (imported and run)", "cases": cases}


def main():
    with tempfile.TemporaryDirectory() as tmp:
        fixtures = {
            "rng_diag_seed42.json": rng_diag(tmp),
            "host_u_stream.json": host_u(tmp),
            "dgp_series.json": dgp(tmp),
            "dgp_scenarios.json": dgp_scenarios(tmp),
        }
    fixtures["systematic_resample.json"] = systematic()
    for name, obj in fixtures.items():
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    sys.exit(main())
