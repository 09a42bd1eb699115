#!/usr/bin/env python
"""Benchmark: pair-moves/s of batched dense spherical parallel tempering.

Workload (one B200 per rank): 256 independent disorder samples of the
fully connected complex 2+4 p-spin model, N drawn from {24, 32, 48, 64} by
splitmix64(2024) (N_k = {24,32,48,64}[z_k mod 4]), seeds 1000 + 256*rank + k,
J = 2, alpha = 0.5 (unit-variance couplings per family), NT = 24 geometric
temperatures in [0.2, 1.6], nrep = 4 replicas per temperature (96 per
sample), exchange after every sweep, FP64 resync every 1024 sweeps.  A step
is `--sweeps-per-step` sweeps (each followed by the exchange) of all 256
samples.  Synthetic inputs: the disorder is generated on the device from the
seeds, as the reference generates it; its per-site sweep lists (several GB)
exceed the 126 MB L2, so no flush is needed between steps.

Lines (rank 0, one JSON line):
  default           the engine: device-resident PT (pspin_pt_run); `e2e` is
                    the reference's driver loop through the C ABI with pinned
                    host buffers (H2D betas, sweep, D2H energies/counters,
                    exchange on the host) every sweep.
  --impl reference  the CPU transcription of the reference sweep (oracle port,
                    FP64, reference loop structure) on the host cores.

Multi-GPU: one process per GPU (torchrun); every rank runs its own 256
samples (weak scaling, no data-path collective); time is the max over ranks.

--workload learned (not the default line): the learned-proposal PT
configuration (dense N=64, uniform FMC gamma=0.1, 24 temperatures geometric
in [0.2, 1.6], 4 replicas each, 64 samples): plain PT with recording, GPU
training of the proposal network, plain equilibration, then interleaved
ABBA blocks of each proposal at its autotuned block shape, reporting
tau_int of E and q and the tau_int-corrected independent samples per second
at slot 19 (T = 0.28714, the grid point nearest 0.3) for both
(cuda_pspin_b200.learned_study).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CLASSES = (24, 32, 48, 64)
NT, NREP_T = 24, 4
TMIN, TMAX = 0.2, 1.6
N_SAMPLES = 256


def splitmix64(state: int):
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


def workload(n_samples: int = N_SAMPLES, rank: int = 0):
    st = 2024
    Ns = []
    for _ in range(n_samples):
        st, z = splitmix64(st)
        Ns.append(N_CLASSES[z % 4])
    seeds = [1000 + n_samples * rank + k for k in range(n_samples)]
    return Ns, seeds


def flops_per_move(N: int) -> float:
    """Algorithmic FLOPs of one pair-move, F = 20*W4 + 4*W2 + 64, fully
    connected: W4 = A(8/N - 12/(N(N-1))) with A = C(N,4) (= 2C(N-2,3)+C(N-2,2)),
    W2 = P(4/N - 2/(N(N-1))) with P = C(N,2) off-diagonal pairs."""
    A = N * (N - 1) * (N - 2) * (N - 3) / 24.0
    Pp = N * (N - 1) / 2.0
    W4 = A * (8.0 / N - 12.0 / (N * (N - 1)))
    W2 = Pp * (4.0 / N - 2.0 / (N * (N - 1)))
    return 20.0 * W4 + 4.0 * W2 + 64.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_engine(args, rank, world, device, dist):
    import torch
    import cuda_pspin_b200 as ps

    Ns, seeds = workload(args.samples, rank)
    T, beta = ps.temperature_schedule(NT, TMIN, TMAX, True)
    cfgs = [ps.default_config(N=N, nrep=NT * NREP_T, seed=s, fmc_mode=0, T=float(T[0]))
            for N, s in zip(Ns, seeds)]
    t_setup = time.perf_counter()
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else None
    opts = ps.make_options(resync_every=1024, warps_per_unit=shape[0] if shape else 0,
                           cluster_size=(shape[1] if shape[1] > 0 else -1) if shape else 0,
                           replicas_per_lane=shape[2] if shape and len(shape) > 2 else 0)
    eng = ps.Engine(cfgs, ps.PSPIN_DENSE, opts)
    t_setup = time.perf_counter() - t_setup
    eng.pt_init(NT, NREP_T, beta, 1)
    sps = args.sweeps_per_step
    moves_per_sweep = sum(NT * NREP_T * (N // 2) for N in Ns)
    flops_per_sweep = sum(NT * NREP_T * (N // 2) * flops_per_move(N) for N in Ns)
    # the library's counts: the same algorithmic F (from the samples' masks)
    # and the FP32 operations its field kernels execute on these site lists
    alg_flops, exec_flops = eng.sweep_work()
    assert abs(alg_flops - flops_per_sweep) <= 1e-9 * flops_per_sweep, (alg_flops, flops_per_sweep)
    entries = sum(eng.info(k).site_entries for k in range(len(Ns)))

    # ---- device-resident PT (value) -------------------------------------------
    for _ in range(args.warmup):
        eng.pt_run(sps)
    # block shape by the engine's autotuner (state restored after its trials),
    # then one more step so the PT graph is captured with that shape
    tuned_table = None
    if shape:
        tuned_w, tuned_c = shape[:2]
        tuned_k = shape[2] if len(shape) > 2 else 1
    else:
        tuned_w, tuned_c, tuned_k, tuned_ms = eng.autotune_lanes(2)
        # ms per sweep of every shape the tuner ran: "K,C,W" -> ms
        tuned_table = {f"{k + 1},{c},{w}": round(float(tuned_ms[k, ci, wi]), 3)
                       for k in range(3) for ci, c in enumerate((0, 1, 2, 4, 8, 16))
                       for wi, w in enumerate((1, 2, 4, 8)) if tuned_ms[k, ci, wi] > 0}
    eng.pt_run(sps)
    eng.get_profile()                  # zero the launch counters
    ext = torch.cuda.ExternalStream(eng.stream_ptr(), device=device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    clocks = ClockSampler(device)
    clocks.start()
    time.sleep(0.3)
    ev0.record(ext)
    for _ in range(args.steps):
        eng.pt_run(sps)                # CUDA-graph replays of 32 PT steps
    ev1.record(ext)
    torch.cuda.synchronize(device)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    _, _, launches = eng.get_profile()
    # per-launch sweep-kernel time for the roofline: one more step with the
    # library's own CUDA events around every sweep launch (direct launches)
    eng.set_profiling(True)
    eng.pt_run(sps)
    kern_ms, sweep_launches, _ = eng.get_profile()
    eng.set_profiling(False)
    if dist:
        t = torch.tensor([ms], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_moves = moves_per_sweep * sps * args.steps * world
    value = total_moves / (ms * 1e-3)

    # ---- roofline of the sweep kernel (FP32 CUDA-core pipe) ---------------------
    peak = ps.fp32_peak_tflops()
    sweeps_per_launch = 1   # pt_freq = 1: one sweep kernel launch per sweep
    per_launch_ms = kern_ms / max(sweep_launches, 1)
    achieved = flops_per_sweep * sweeps_per_launch / (per_launch_ms * 1e-3) / 1e12
    traffic = None
    tf = os.path.join(ROOT, "profiles", "sweep_dense_batched_traffic.json")
    if os.path.exists(tf):
        try:
            rec = json.load(open(tf))
            # the capture of the kernel this launch ran: cluster split, one CTA,
            # or K replicas per lane
            if tuned_k > 1:
                rec = rec.get(f"replicas_per_lane_{tuned_k}", {})
            elif tuned_c == 1 and "one_cta_kernel" in rec:
                rec = rec["one_cta_kernel"]
            traffic = None if tuned_c == 0 else rec.get("bytes_per_launch")
        except Exception:
            traffic = None
    executed = exec_flops * sweeps_per_launch / (per_launch_ms * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": "FMA-loop probe on this GPU (pspin_fp32_peak)",
            "kernel_ms_per_launch": per_launch_ms,
            "flops_per_launch": flops_per_sweep,
            "executed_flops_per_launch": exec_flops * sweeps_per_launch,
            "executed_achieved": executed, "executed_frac": executed / peak,
            "note": "achieved/frac count the reference method's F = 20 W4 + 4 W2 + 64 FLOPs per pair-move; "
                    "the local-field kernels execute about 4 per quartet term and replica "
                    "(executed_*, counted from the site lists by pspin_sweep_work)",
            "site_entries": entries}

    # ---- FP64 resync (every 1024 sweeps): its cost, amortised over its period
    eng.set_profiling(False)
    ev_r0 = torch.cuda.Event(enable_timing=True)
    ev_r1 = torch.cuda.Event(enable_timing=True)
    eng.resync()                       # warm
    ev_r0.record(ext)
    for _ in range(3):
        eng.resync()
    ev_r1.record(ext)
    torch.cuda.synchronize(device)
    resync_ms = ev_r0.elapsed_time(ev_r1) / 3
    sweep_ms = ms / (args.steps * sps)
    resync = {"ms": resync_ms, "every_sweeps": 1024, "share_of_loop": resync_ms / (resync_ms + 1024 * sweep_ms),
              "value_with_resync": moves_per_sweep * world / ((sweep_ms + resync_ms / 1024) * 1e-3)}

    # ---- end to end: the reference's driver loop through the C ABI -------------------
    R_tot = eng.n_replicas
    pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
    b_host = pin(R_tot, torch.float64)
    E_host = pin(R_tot, torch.float64)
    a_host = pin(R_tot, torch.int64)
    p_host = pin(R_tot, torch.int64)
    S = len(Ns)
    rep_off = np.arange(S, dtype=np.int64) * (NT * NREP_T)
    perm = np.tile(np.arange(NT * NREP_T, dtype=np.int32), (S, 1))
    st = np.array([((s + 5000) & 0xFFFFFFFF) << 16 | 0x330E for s in seeds], dtype=np.uint64)
    exa = np.zeros((S, NT - 1), np.int64)
    exp_ = np.zeros((S, NT - 1), np.int64)
    lib = eng._lib

    def rebuild_betas():
        b = np.empty((S, NT * NREP_T))
        b[np.arange(S)[:, None], perm] = np.repeat(beta, NREP_T)[None, :]
        b_host[:] = b.ravel()

    def e2e_sweep():
        lib.pspin_set_betas(eng._h, ps._ptr(b_host))
        lib.pspin_sweep(eng._h, 1)
        lib.pspin_get_results(eng._h, ps._ptr(E_host), ps._ptr(a_host), ps._ptr(p_host))
        # the reference's host exchange (parallel_tempering.cu:316-352), in the library, betas rebuilt in place
        ps.exchange_host(beta, E_host, rep_off, perm, st, exa, exp_, b_host)

    rebuild_betas()
    for _ in range(args.warmup):
        e2e_sweep()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(args.steps * sps):
        e2e_sweep()
    torch.cuda.synchronize(device)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": total_moves / e2e_s, "unit": "pair-moves/s", "h2d_bytes_per_step": 8 * R_tot * sps,
           "d2h_bytes_per_step": 24 * R_tot * sps,
           "loop": "per sweep: pspin_set_betas (H2D, pinned) + pspin_sweep + pspin_get_results (D2H, pinned) "
                   "+ pspin_exchange_host (drand48, parallel_tempering.cu:316-352, OpenMP over samples)"}
    eng.free()

    out = {
        "metric": "pair-moves/s", "value": value, "unit": "pair-moves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 running energy, FP64 resync)", "data": "synthetic",
        "config": {"workload": f"batched dense spherical PT: {S} samples, N from {{24,32,48,64}} "
                               f"(counts {[Ns.count(n) for n in N_CLASSES]}), FC, NT={NT} geometric "
                               f"[{TMIN},{TMAX}], nrep={NREP_T}, exchange every sweep",
                   "samples_per_gpu": S, "replicas_per_sample": NT * NREP_T, "sweeps_per_step": sps,
                   "pair_moves_per_sweep_per_gpu": moves_per_sweep,
                   "l2": f"inputs exceed L2: {entries * 8 / 1e9:.2f} GB of site lists per GPU (no flush)",
                   "parallelism": f"samples sharded, {world} GPU(s), no collective",
                   "block_shape": {"warps_per_cta": tuned_w, "ctas_per_replica_block": tuned_c,
                                   "replicas_per_lane": tuned_k,
                                   "chosen_by": "--shape" if shape else "pspin_autotune_lanes (2 sweeps per shape)",
                                   "ms_per_sweep_by_replicas_per_lane_cluster_warps": tuned_table},
                   "launch": "sweep + exchange per PT step, replayed as CUDA graphs of 32 steps",
                   "setup_s": t_setup},
        "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": clk, "resync": resync,
    }
    # whole 2^14-sweep job of this workload from the measured parts: set-up,
    # the e2e per-sweep loop, and a resync every 1024 sweeps
    job_sweeps = 1 << 14
    job_s = t_setup + job_sweeps * (e2e_s / (args.steps * sps)) + (job_sweeps // 1024) * resync_ms * 1e-3
    out["e2e"]["job_projection"] = {"sweeps": job_sweeps, "seconds": job_s,
                                    "pair_moves_per_s": moves_per_sweep * job_sweeps / job_s,
                                    "parts": "set-up + 2^14 x (e2e seconds per sweep) + 16 resyncs"}
    return out


def cpu_port_rate(args, sample_classes=True):
    """The oracle's CPU transcription of the reference sweep on one sample per
    N class; returns pair-moves/s extrapolated to the workload's N mix."""
    import oracle
    Ns, seeds = workload(args.samples, 0)
    T = np.array([TMAX * (TMIN / TMAX) ** (t / (NT - 1)) for t in range(NT)])
    beta = 1.0 / T
    per_class, threads = oracle.cpu_sweep_rate(list(N_CLASSES), [seeds[0] + 7 * i for i in range(4)], NT, NREP_T,
                                               beta, sweeps=1, nthreads=args.cpu_threads)
    t_class = dict(zip(N_CLASSES, per_class))
    sweep_s = sum(t_class[N] for N in Ns)
    moves = sum(NT * NREP_T * (N // 2) for N in Ns)
    return moves / sweep_s, threads, t_class


def run_learned(args, rank, world):
    """The learned-proposal configuration on one GPU (rank 0; the other ranks
    exit): one JSON line with both proposals' tau_int and independent
    samples per second at slot 19."""
    if rank != 0:
        return 0
    import torch
    from cuda_pspin_b200 import learned_study
    torch.cuda.set_device(0)
    study_args = argparse.Namespace(
        N=64, samples=64, NT=NT, nrep=NREP_T, gamma=0.1, Tmin=TMIN, Tmax=TMAX, slot=19, seed0=42,
        train_sweeps=1 << 14, equilibrate=args.equilibrate, measure_sweeps=1 << 14, blocks=16,
        capacity=1 << 22, record_prob=0.01, train_steps=3000, batch=8192, lr=2e-3, net_seed=1, out="")
    clocks = ClockSampler(0)
    clocks.start()
    res = learned_study.run(study_args)
    clk = clocks.stop()
    p, l = res["plain"], res["learned"]
    keep = ("tau_E", "tau_E_err", "tau_q", "tau_q_err", "sweeps_per_s", "indep_E_per_s", "indep_q_per_s",
            "E_per_N", "E_per_N_err", "acceptance_all_T")
    line = {"metric": "tau_int-corrected independent E samples/s at T=0.28714 (slot 19)",
            "value": l["indep_E_per_s"], "unit": "samples/s", "n_gpus": 1, "steps": study_args.blocks,
            "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 running energy; BF16 network weights, FP32 accumulate)", "data": "synthetic",
            "config": {"workload": "learned-proposal PT: 64 samples, dense N=64, uniform FMC gamma=0.1, NT=24 "
                                   "geometric [0.2,1.6], nrep=4, exchange every sweep",
                       "train_sweeps": study_args.train_sweeps, "equilibrate_sweeps": study_args.equilibrate,
                       "measure_sweeps_per_proposal": study_args.measure_sweeps,
                       "blocks_per_proposal": study_args.blocks, "block_shapes": res["block_shapes"]},
            "plain": {k: p[k] for k in keep}, "learned": {k: l[k] for k in keep},
            "gain_E": res["gain_E"], "gain_q": res["gain_q"], "gain_q2": res["gain_q2"],
            "E_learned_minus_plain": res["E_diff_mean"], "E_diff_err": res["E_diff_err"],
            "E_diff_sigma": res["E_diff_sigma"],
            "plain_block_means_first_last": [res["plain_block_means"][0], res["plain_block_means"][-1]],
            "training": {k: res["training"][k] for k in ("records_seen", "train_s", "loss_start", "loss_end")},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--samples", type=int, default=N_SAMPLES)
    ap.add_argument("--sweeps-per-step", type=int, default=16)
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="", help="W,C[,K]: warps per CTA, CTAs per replica block, replicas per "
                                                "lane (skips the autotuner; for profiling a fixed kernel shape)")
    ap.add_argument("--workload", default="batched", choices=["batched", "learned"])
    ap.add_argument("--equilibrate", type=int, default=1 << 15,
                    help="learned workload: plain PT sweeps between training and measuring")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        rates = []
        threads = 1
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r, threads, t_class = cpu_port_rate(args)
            rates.append(r)
        wall = time.perf_counter() - t0
        v = float(np.median(rates))
        Ns, _ = workload(args.samples, 0)
        line = {"metric": "pair-moves/s", "value": v, "unit": "pair-moves/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": f"batched dense spherical PT: {args.samples} samples, N from {{24,32,48,64}}, "
                                       f"FC, NT={NT}, nrep={NREP_T}", "samples_per_gpu": args.samples},
                "cpu_baseline": {"value": v, "unit": "pair-moves/s", "cores": threads, "kind": "port",
                                 "sample": "per step one sweep of one sample per N class (96 replicas each), "
                                           "extrapolated to the workload's N mix; per-class s/sweep "
                                           + json.dumps({str(k): round(x, 4) for k, x in t_class.items()})},
                "e2e": {"value": v, "unit": "pair-moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "learned":
        return run_learned(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = tdist
    torch.cuda.set_device(local)
    out = run_engine(args, rank, world, local, dist)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            rate, threads, t_class = cpu_port_rate(args)
            out["cpu_baseline"] = {"value": rate, "unit": "pair-moves/s", "cores": threads, "kind": "port",
                                   "sample": "one sweep of one sample per N class (96 replicas each), "
                                             "extrapolated to the workload's N mix"}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
