"""Statistical parity with the reference binary over 64 disorder samples.

The engine (pspin_pt -batch 64) and the reference's parallel_tempering
(rebuilt for sm_100a, oracle/_ref/, one process per sample) run the same PT
on the same 64 disorder samples (seeds 100..163, same couplings and initial
amplitudes bit for bit).  The trajectories differ (the engine shares the pair
schedule among a sample's replicas and uses its own move streams), so the
comparison is statistical and paired: for every temperature, the mean over
samples of (engine - reference) of the second-half averages of E/N, the
Metropolis acceptance, the exchange rate and <q^2> is compared with its
standard error (z-score).  Checked: every |z| < 3.5 (six temperatures x four
observables) and at least 80 % of them within 2 sigma.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cuda_pspin_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
N, NT, NREP, ITER, SAVE = 12, 6, 4, 4096, 32
SAMPLES = 64
FLAGS = ["-N", str(N), "-Tmax", "1.5", "-Tmin", "0.3", "-NT", str(NT), "-log_temp", "-nrep", str(NREP),
         "-iter", str(ITER), "-pt_freq", "1", "-save_freq", str(SAVE)]


def observables(d):
    """Second-half averages per temperature: E/N, acceptance, exchange rate, <q^2>."""
    ea = np.loadtxt(os.path.join(d, "energy_accept.txt"))
    half = ea[:, 0] > ITER / 2
    E = np.zeros(NT)
    A = np.zeros(NT)
    for t in range(NT):
        rows = ea[half & (ea[:, 1] == t)]
        E[t] = rows[:, 3::2].mean()
        A[t] = rows[:, 4::2].mean()
    ex = np.loadtxt(os.path.join(d, "exchanges.txt"))
    X = np.zeros(NT)
    for t in range(NT - 1):
        rows = ex[(ex[:, 0] > ITER / 2) & (ex[:, 1] == t)]
        X[t] = rows[:, 4].sum() / rows[:, 5].sum()
    raw = np.fromfile(os.path.join(d, "configs.bin"), dtype=np.uint8)
    hdr = np.frombuffer(raw[:12].tobytes(), np.int32)
    assert tuple(hdr) == (N, NT, NREP)
    rec = 4 + NT * NREP * 2 * N * 8
    body = raw[12:]
    nsnap = len(body) // rec
    Q = np.zeros(NT)
    for sidx in range(nsnap):
        chunk = body[sidx * rec + 4:(sidx + 1) * rec]
        a = np.frombuffer(chunk.tobytes(), np.float64).reshape(NT, NREP, N, 2)
        z = a[..., 0] + 1j * a[..., 1]
        for t in range(NT):
            qs = [np.real(np.sum(z[t, r1] * np.conj(z[t, r2]))) / N
                  for r1 in range(NREP) for r2 in range(r1 + 1, NREP)]
            Q[t] += np.mean(np.square(qs))
    Q /= max(nsnap, 1)
    return E, A, X, Q


def test_engine_matches_reference_statistics(tmp_path):
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    p = subprocess.run([os.path.join(BIN, "pspin_pt"), *FLAGS, "-seed", "100", "-label", "0",
                        "-batch", str(SAMPLES)], cwd=ours, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    for k in range(SAMPLES):
        p = subprocess.run([os.path.join(REF, "parallel_tempering"), *FLAGS, "-seed", str(100 + k),
                            "-label", str(k)], cwd=ref, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-2000:]
    dirs_o = sorted(os.listdir(ours / "data"))
    dirs_r = sorted(os.listdir(ref / "data"))
    assert dirs_o == dirs_r and len(dirs_o) == SAMPLES
    obs_o = np.array([observables(str(ours / "data" / d)) for d in dirs_o])   # [S, 4, NT]
    obs_r = np.array([observables(str(ref / "data" / d)) for d in dirs_r])
    diff = obs_o - obs_r
    mean = diff.mean(axis=0)
    se = diff.std(axis=0, ddof=1) / np.sqrt(SAMPLES)
    valid = np.ones_like(mean, dtype=bool)
    valid[2, NT - 1] = False                  # no exchange above the coldest temperature
    z = np.where(valid, mean / np.where(se > 0, se, 1.0), 0.0)
    report = {name: np.round(z[i], 2).tolist() for i, name in enumerate(["E/N", "acc", "exchange", "q2"])}
    print("paired z-scores per temperature:", report)
    print("engine E/N per T:", np.round(obs_o[:, 0].mean(axis=0), 4).tolist())
    print("reference E/N per T:", np.round(obs_r[:, 0].mean(axis=0), 4).tolist())
    assert np.all(np.abs(z[valid]) < 3.5), report
    assert np.mean(np.abs(z[valid]) < 2.0) >= 0.8, report
