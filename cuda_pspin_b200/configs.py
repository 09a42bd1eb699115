"""The engine on the benchmark configurations beside the reference's sm_100a
rebuild (its numbers, when present, from profiles/reference_sm100_timing.json,
written by tests/golden/time_reference.py on the same kind of GPU).

  1  dense spherical PT, N=32, FMC uniform gamma=0.1, NT=20 geometric in
     [0.2, 1.6], nrep 4, seed 42 (one sample)
  2  sparse cube PT, N=512, FMC comb gamma=1, NT=32, nrep 4, seed 42
  4  dense spherical MC, N=128 fully connected, 64 replicas at T=0.5
  5  dense spherical PT, N=64, FMC uniform gamma=0.1, NT=24, nrep 4:
     one sample (seed 42, the reference's run) and 64 samples (seeds 42..105)
(3, the batched workload, is bench.py's.)

Each run: set-up, a few warm-up sweeps, the block-shape autotuner (block
shape and replicas per lane, pspin_autotune_lanes), then a
timed run of device-resident sweeps (PT cycles replayed as CUDA graphs) with
the wall clock around the synchronous calls.  Rate = replicas x N/2 x sweeps
/ seconds (pair-moves/s), the reference's unit.

--precision runs configuration 4 for 2^12 sweeps with the running energy
resynchronised every 256 sweeps from the split-BF16 tensor-core contraction
and reports, per resync, the FP32 accumulation drift and, at the end, the
running and tensor-core energies against the FP64 energies of the same
amplitudes.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from . import (Engine, PSPIN_DENSE, PSPIN_SPARSE, RESYNC_TC, FIELDS_TC_BF16X3, default_config, make_options,
               temperature_schedule)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_KEYS = {"1": "config1_dense_pt_n32_fmc2", "2": "config2_sparse_pt_n512_comb", "4": "config4_dense_mc_n128",
            "5": "config5_dense_pt_n64_fmc2"}


def _pt_engine(N, seeds, NT, nrep, variant, fmc, gamma, shape, Tmin=0.2, Tmax=1.6, stream=False):
    cfgs = []
    for s in seeds:
        c = default_config(N=N, nrep=NT * nrep, seed=s, fmc_mode=fmc)
        c.gamma = gamma
        cfgs.append(c)
    t0 = time.perf_counter()
    eng = Engine(cfgs, variant, _options(shape, disorder_stream=stream))
    setup = time.perf_counter() - t0
    _, betas = temperature_schedule(NT, Tmin, Tmax, True)
    eng.pt_init(NT, nrep, betas, 1)
    return eng, setup


def _options(shape, **kw):
    w, c = shape[:2] if shape else (0, None)
    c = 0 if c is None else (-1 if c == 0 else c)      # 0 from the autotuner: the list-resident kernel
    k = shape[2] if shape and len(shape) > 2 else 0
    return make_options(quiet=True, warps_per_unit=w, cluster_size=c, replicas_per_lane=k, **kw)


def _timed(eng, run, sweeps, warmup, tune_sweeps, shape):
    run(warmup)
    if shape:
        w, c = shape[:2]
        k = shape[2] if len(shape) > 2 else 1
    else:
        w, c, k, ms = eng.autotune_lanes(tune_sweeps)
    run(warmup)
    t0 = time.perf_counter()
    run(sweeps)
    return time.perf_counter() - t0, w, c, k


def measure(config: str, sweeps: int | None = None, shape=None, stream: bool = False) -> dict:
    """stream: sparse couplings from per-quartet counter-based normals
    (options.disorder_stream) instead of the reference's 2*C(N,4) cuRAND
    normals (45 GB on the device at N=512 during set-up); same law and
    kernels, not the reference's values."""
    if config == "1":
        eng, setup = _pt_engine(32, [42], 20, 4, PSPIN_DENSE, 2, 0.1, shape)
        sweeps = sweeps or 4096
        run = eng.pt_run
    elif config == "2":
        eng, setup = _pt_engine(512, [42], 32, 4, PSPIN_SPARSE, 1, 1.0, shape, stream=stream)
        sweeps = sweeps or 4096
        run = eng.pt_run
    elif config == "4":
        c = default_config(N=128, nrep=64, seed=42, fmc_mode=0, T=0.5)
        t0 = time.perf_counter()
        eng = Engine(c, PSPIN_DENSE, _options(shape))
        setup = time.perf_counter() - t0
        eng.fill_betas(2.0)
        sweeps = sweeps or 64
        run = eng.sweep
    elif config == "5":
        eng, setup = _pt_engine(64, [42], 24, 4, PSPIN_DENSE, 2, 0.1, shape)
        sweeps = sweeps or 2048
        run = eng.pt_run
    elif config == "5x64":
        eng, setup = _pt_engine(64, list(range(42, 106)), 24, 4, PSPIN_DENSE, 2, 0.1, shape)
        sweeps = sweeps or 1024
        run = eng.pt_run
    else:
        raise ValueError(config)
    moves = sum(N * R // 2 for N, R in zip(eng.Ns, eng.Rs))
    chains = sum(eng.Rs)
    secs, w, cl, k = _timed(eng, run, sweeps, warmup=8 if config != "4" else 2,
                         tune_sweeps=2 if config == "4" else 8, shape=shape)
    eng.free()
    rate = moves * sweeps / secs
    # latency-bound configurations: time per move along one replica's chain
    out = {"config": config, "sweeps": sweeps, "seconds": secs, "pair_moves_per_s": rate,
           "chains": chains, "ns_per_move_per_chain": 1e9 * chains / rate,
           "warps_per_cta": w, "ctas_per_replica_block": cl, "replicas_per_lane": k, "setup_s": setup}
    ref = os.path.join(ROOT, "profiles", "reference_sm100_timing.json")
    key = REF_KEYS.get(config)
    if key and os.path.exists(ref):
        r = json.load(open(ref)).get(key)
        if r:
            out["reference_pair_moves_per_s"] = r["pair_moves_per_s"]
            out["reference_ns_per_move_per_chain"] = 1e9 * chains / r["pair_moves_per_s"]
            out["speedup_vs_reference"] = out["pair_moves_per_s"] / r["pair_moves_per_s"]
    return out


def precision(sweeps: int = 1 << 12, every: int = 256) -> dict:
    c = default_config(N=128, nrep=64, seed=42, fmc_mode=0, T=0.5)
    eng = Engine(c, PSPIN_DENSE, make_options(quiet=True, resync_every=every, resync_method=RESYNC_TC))
    eng.fill_betas(2.0)
    w, cl, _ = eng.autotune(2)
    drifts = []
    t0 = time.perf_counter()
    for _ in range(sweeps // every):
        eng.sweep(every)                       # ends on a resync
        drifts.append(float(eng.resync_drift().max() / c.N))
    secs = time.perf_counter() - t0
    E_run, _, _ = eng.get_results()
    e2, e4 = eng.split_energies()            # FP64, same amplitudes
    E64 = e2 + e4
    _, E_tc = eng.local_fields(0, FIELDS_TC_BF16X3)
    eng.free()
    rel = lambda a: float(np.max(np.abs(a - E64) / np.abs(E64)))
    return {"config": "4-precision", "sweeps": sweeps, "resync_every": every, "seconds": secs,
            "warps_per_cta": w, "ctas_per_replica_block": cl,
            "max_fp32_drift_per_site_between_resyncs": drifts,
            "final_E_per_site_fp64_mean": float(E64.mean() / c.N),
            "final_running_vs_fp64_max_rel": rel(E_run), "final_tc_vs_fp64_max_rel": rel(np.asarray(E_tc)),
            "final_running_vs_fp64_max_abs_per_site": float(np.max(np.abs(E_run - E64)) / c.N)}


def fields(repeats: int = 5) -> dict:
    """All-site local fields of configuration 4 (N=128 FC, 64 replicas): the
    split-BF16 tcgen05 contraction against the FP64 table sum, time and error."""
    from . import FIELDS_FP64
    c = default_config(N=128, nrep=64, seed=42, fmc_mode=0, T=0.5)
    eng = Engine(c, PSPIN_DENSE, make_options(quiet=True))
    eng.local_fields(0, FIELDS_TC_BF16X3)                      # operand preparation (once per sample)
    t0 = time.perf_counter()
    for _ in range(repeats):
        h_tc, e_tc = eng.local_fields(0, FIELDS_TC_BF16X3)
    t_tc = (time.perf_counter() - t0) / repeats
    t0 = time.perf_counter()
    h64, e64 = eng.local_fields(0, FIELDS_FP64)
    t_64 = time.perf_counter() - t0
    eng.free()
    rel = float(np.abs(h_tc - h64).max() / np.abs(h64).max())
    return {"config": "4-fields", "N": 128, "replicas": 64, "tc_ms_per_call": t_tc * 1e3, "fp64_ms_per_call": t_64 * 1e3,
            "fields_max_err_rel_to_max": rel,
            # per site: the initial random state has energies near zero, so a relative error says little
            "energy_max_abs_err_per_site": float(np.max(np.abs(e_tc - e64)) / 128)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--configs", default="1,2,4,5,5x64")
    ap.add_argument("--precision", action="store_true")
    ap.add_argument("--fields", action="store_true", help="tensor-core vs FP64 all-site fields at configuration 4")
    ap.add_argument("--sweeps", type=int, default=0, help="timed sweeps (0: the configuration's default)")
    ap.add_argument("--shape", default="", help="W,C[,K]: warps per CTA, CTAs per replica block, replicas per lane "
                                                "(skips the autotuner)")
    ap.add_argument("--disorder-stream", action="store_true",
                    help="configuration 2: streamed sparse couplings (no 45 GB set-up buffer)")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    shape = tuple(int(x) for x in a.shape.split(",")) if a.shape else None
    res = [measure(k, a.sweeps or None, shape, a.disorder_stream) for k in a.configs.split(",") if k]
    if a.precision:
        res.append(precision())
    if a.fields:
        res.append(fields())
    for r in res:
        print(json.dumps(r))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
            f.write("\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
