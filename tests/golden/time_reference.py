"""Times the reference's own sweep, rebuilt for sm_100a (oracle/_ref/ref_bench:
its mc_sweep_pt / mc_sparse_sweep_pt with the host exchange of
parallel_tempering.cu:316-352 after every sweep, cudaEvent timing as in its
bench_pt_scaling.cu:73-165), on the configurations of the benchmark suite,
and writes a JSON summary:

    python tests/golden/time_reference.py --out profiles/reference_sm100_timing.json

The batched workload (256 samples, N in {24,32,48,64}, NT=24, nrep=4, FC) is
run by the reference as 256 separate processes, so its rate is the workload's
pair-moves per sweep divided by the sum of the per-sample sweep times.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")


def run(args: list[str], timeout: int = 900) -> dict:
    out = subprocess.run([BENCH, *args], capture_output=True, text=True, timeout=timeout, check=True).stdout
    last = [ln for ln in out.strip().splitlines() if ln and ln[0].isdigit()][-1].split()
    N, NT, nr, sweeps = (int(x) for x in last[:4])
    return {"N": N, "NT": NT, "nrepT": nr, "sweeps": sweeps, "ms_total": float(last[4]),
            "ms_per_sweep": float(last[5]), "pair_moves_per_s": float(last[6]), "args": args}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--skip-sparse512", action="store_true")
    a = ap.parse_args()
    import bench
    res = {"what": "reference cuda_pspin rebuilt for sm_100a (its Makefile flags, -arch replaced), "
                   "kernel launches + cudaDeviceSynchronize + host exchange per sweep"}
    classes = {}
    for N, sweeps in [(24, 32), (32, 32), (48, 8), (64, 4)]:
        classes[N] = run(["dense", "-N", str(N), "-NT", "24", "-nrepT", "4", "-sweeps", str(sweeps), "-warmup", "1",
                          "-seed", str(1000 + N)])
    Ns, _ = bench.workload()
    sweep_s = sum(classes[N]["ms_per_sweep"] for N in Ns) * 1e-3
    moves = sum(24 * 4 * (N // 2) for N in Ns)
    res["batched_dense_pt_256"] = {"per_class": classes, "pair_moves_per_s": moves / sweep_s,
                                   "s_per_sweep_all_samples": sweep_s}
    res["config1_dense_pt_n32_fmc2"] = run(["dense", "-N", "32", "-NT", "20", "-nrepT", "4", "-sweeps", "64",
                                            "-warmup", "2", "-fmc", "2", "-gamma", "0.1", "-seed", "42"])
    res["config4_dense_mc_n128"] = run(["dense", "-N", "128", "-NT", "2", "-nrepT", "32", "-sweeps", "2",
                                        "-warmup", "1", "-Tmin", "0.5", "-Tmax", "0.5", "-exchange", "0"])
    res["config5_dense_pt_n64_fmc2"] = run(["dense", "-N", "64", "-NT", "24", "-nrepT", "4", "-sweeps", "8",
                                            "-warmup", "1", "-fmc", "2", "-gamma", "0.1", "-seed", "42"])
    if not a.skip_sparse512:
        res["config2_sparse_pt_n512_comb"] = run(["sparse", "-N", "512", "-NT", "32", "-nrepT", "4", "-sweeps",
                                                  "64", "-warmup", "4", "-fmc", "1", "-gamma", "1.0", "-seed", "42"],
                                                 timeout=1800)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
