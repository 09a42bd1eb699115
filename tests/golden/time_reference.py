"""Times the reference's own sweep, rebuilt for sm_100a (oracle/_ref/ref_bench:
its mc_sweep_pt / mc_sparse_sweep_pt with the host exchange of
parallel_tempering.cu:316-352 after every sweep, cudaEvent timing as in its
bench_pt_scaling.cu:73-165), on the configurations of the benchmark suite,
and writes a JSON summary:

    python tests/golden/time_reference.py --out profiles/reference_sm100_timing.json

The batched workload (256 samples, N in {24,32,48,64}, NT=24, nrep=4, FC) is
run by the reference as 256 separate processes, so its rate is the workload's
pair-moves per sweep divided by the sum of the per-sample sweep times.

    python tests/golden/time_reference.py --workload-samples 64 --out profiles/reference_sm100_batched.json

times the first K samples of that workload exactly (each its own N and seed,
as bench.py builds them; 4 sweeps each after a warm-up sweep) on the
reference rebuild, and the CPU port (oracle, FP64, OpenMP over replicas) on
the first `--cpu-per-class` samples of each N class, with the GPU clocks
sampled during the reference runs.
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


def workload_subset(K: int, cpu_per_class: int) -> dict:
    """The first K samples of bench.py's batched workload on the reference
    rebuild, exactly; the CPU port on cpu_per_class samples of each N class."""
    import time
    import numpy as np
    import bench
    import oracle
    Ns, seeds = bench.workload()
    clocks = bench.ClockSampler(0)
    clocks.start()
    per = []
    t0 = time.perf_counter()
    for N, seed in zip(Ns[:K], seeds[:K]):
        r = run(["dense", "-N", str(N), "-NT", "24", "-nrepT", "4", "-sweeps", "4", "-warmup", "1", "-seed", str(seed)])
        per.append({"N": N, "seed": seed, "ms_per_sweep": r["ms_per_sweep"]})
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    moves = sum(24 * 4 * (N // 2) for N in Ns[:K])
    sweep_s = sum(x["ms_per_sweep"] for x in per) * 1e-3
    ref = {"samples": K, "counts_per_N": {str(n): Ns[:K].count(n) for n in bench.N_CLASSES},
           "sweeps_per_sample": 4, "pair_moves_per_s": moves / sweep_s, "s_per_sweep_of_subset": sweep_s,
           "wall_s_incl_init": wall, "per_sample": per, "clocks": clk}
    # CPU port: several samples of each class, extrapolated to the whole workload's N mix
    T = np.array([bench.TMAX * (bench.TMIN / bench.TMAX) ** (t / (bench.NT - 1)) for t in range(bench.NT)])
    t_class, threads = {}, 1
    for N in bench.N_CLASSES:
        picks = [s for n, s in zip(Ns, seeds) if n == N][:cpu_per_class]
        secs, threads = oracle.cpu_sweep_rate([N] * len(picks), picks, bench.NT, bench.NREP_T, 1.0 / T, sweeps=1)
        t_class[N] = {"seeds": picks, "s_per_sweep": secs, "mean": float(np.mean(secs))}
    cpu_sweep_s = sum(t_class[N]["mean"] for N in Ns)
    cpu = {"kind": "port", "threads": threads, "samples_per_class": cpu_per_class, "per_class": t_class,
           "pair_moves_per_s": sum(24 * 4 * (N // 2) for N in Ns) / cpu_sweep_s}
    return {"reference_sm100": ref, "cpu_port": cpu}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--skip-sparse512", action="store_true")
    ap.add_argument("--workload-samples", type=int, default=0,
                    help="time only the first K samples of the batched workload exactly (and the CPU port)")
    ap.add_argument("--cpu-per-class", type=int, default=4)
    a = ap.parse_args()
    import bench
    if a.workload_samples > 0:
        res = {"what": "reference cuda_pspin rebuilt for sm_100a (its Makefile flags, -arch replaced), kernel "
                       "launches + cudaDeviceSynchronize + host exchange per sweep, on the first samples of "
                       "bench.py's batched workload"}
        res.update(workload_subset(a.workload_samples, a.cpu_per_class))
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
        print(json.dumps({k: v for k, v in res["reference_sm100"].items() if k != "per_sample"}))
        print(json.dumps({"cpu_port_pair_moves_per_s": res["cpu_port"]["pair_moves_per_s"]}))
        return 0
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
