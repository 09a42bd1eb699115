"""Statistical parity with the reference binaries over 64 disorder samples.

The engine's drivers (pspin_pt / pspin_pt_sparse -batch 64) and the
reference's parallel_tempering / parallel_tempering_sparse (rebuilt for
sm_100a, oracle/_ref/, one process per sample) run the same PT on the same 64
disorder samples (seeds 100..163, same couplings, sparse selection and
initial amplitudes bit for bit).  The trajectories differ (the engine shares
the pair schedule among a sample's replicas and uses its own move streams),
so the comparison is statistical and paired: for every temperature, the mean
over samples of (engine - reference) of the second-half averages of E/N, the
Metropolis acceptance, the exchange rate, <q^2> and the overlap distribution
P(q) (8 bins over [-1, 1], pooled over the saved configurations and replica
pairs) is compared with its standard error (z-score).

Cases: small dense (N=12) and sparse (N=16, comb) runs, and the dense
benchmark configuration "plain spherical PT" (N=32, uniform FMC with
gamma=0.1, NT=20 geometric temperatures in [0.2, 1.6], nrep=4) at 2048
sweeps.  The bar: no |z| above 4, and at most 10 % of the z-scores outside
2 sigma (5 % expected if the engine samples the reference's law; the
z-scores of neighbouring temperatures are correlated, so their count
fluctuates more than a binomial's).  The count is printed.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cuda_pspin_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
NREP, SAVE = 4, 32
SAMPLES = 64
QBINS = np.linspace(-1.0, 1.0, 9)

CASES = {
    "dense": dict(N=12, NT=6, T=(0.3, 1.5), iter=4096, engine="pspin_pt", ref="parallel_tempering", extra=[]),
    "sparse": dict(N=16, NT=6, T=(0.3, 1.5), iter=4096, engine="pspin_pt_sparse", ref="parallel_tempering_sparse",
                   extra=["-fmc", "1", "-gamma", "1"]),
    "dense_n32_fmc": dict(N=32, NT=20, T=(0.2, 1.6), iter=2048, engine="pspin_pt", ref="parallel_tempering",
                          extra=["-fmc", "2", "-gamma", "0.1"]),
}


def flags(case):
    return ["-N", str(case["N"]), "-Tmax", str(case["T"][1]), "-Tmin", str(case["T"][0]), "-NT", str(case["NT"]),
            "-log_temp", "-nrep", str(NREP), "-iter", str(case["iter"]), "-pt_freq", "1", "-save_freq", str(SAVE)]


def observables(d, N, NT, ITER):
    """Second-half averages per temperature: E/N, acceptance, exchange rate,
    <q^2>, and the P(q) histogram."""
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
    H = np.zeros((NT, len(QBINS) - 1))
    for sidx in range(nsnap):
        chunk = body[sidx * rec + 4:(sidx + 1) * rec]
        a = np.frombuffer(chunk.tobytes(), np.float64).reshape(NT, NREP, N, 2)
        z = a[..., 0] + 1j * a[..., 1]
        for t in range(NT):
            qs = np.array([np.real(np.sum(z[t, r1] * np.conj(z[t, r2]))) / N
                           for r1 in range(NREP) for r2 in range(r1 + 1, NREP)])
            Q[t] += np.mean(np.square(qs))
            H[t] += np.histogram(np.clip(qs, -1.0, 1.0), bins=QBINS)[0]
    Q /= max(nsnap, 1)
    H /= np.maximum(H.sum(axis=1, keepdims=True), 1)
    return np.concatenate([np.stack([E, A, X, Q]), H.T])           # [4 + bins, NT]


def _run_refs(prog, fl, cwd, n, par=4):
    """The reference's one-sample-per-process runs, `par` at a time."""
    procs, k = [], 0
    while k < n or procs:
        while k < n and len(procs) < par:
            procs.append(subprocess.Popen([prog, *fl, "-seed", str(100 + k), "-label", str(k)], cwd=cwd,
                                          stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True))
            k += 1
        p = procs.pop(0)
        _, err = p.communicate(timeout=1800)
        assert p.returncode == 0, err[-2000:]


@pytest.mark.parametrize("variant", ["dense", "sparse", "dense_n32_fmc"])
def test_engine_matches_reference_statistics(tmp_path, variant):
    case = CASES[variant]
    N, NT, ITER = case["N"], case["NT"], case["iter"]
    fl = flags(case) + case["extra"]
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    p = subprocess.run([os.path.join(BIN, case["engine"]), *fl, "-seed", "100", "-label", "0",
                        "-batch", str(SAMPLES)], cwd=ours, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    _run_refs(os.path.join(REF, case["ref"]), fl, ref, SAMPLES)
    dirs_o = sorted(os.listdir(ours / "data"))
    dirs_r = sorted(os.listdir(ref / "data"))
    assert dirs_o == dirs_r and len(dirs_o) == SAMPLES
    obs_o = np.array([observables(str(ours / "data" / d), N, NT, ITER) for d in dirs_o])   # [S, 4 + bins, NT]
    obs_r = np.array([observables(str(ref / "data" / d), N, NT, ITER) for d in dirs_r])
    diff = obs_o - obs_r
    mean = diff.mean(axis=0)
    se = diff.std(axis=0, ddof=1) / np.sqrt(SAMPLES)
    valid = se > 0                              # e.g. P(q) bins that neither side ever fills
    valid[2, NT - 1] = False                    # no exchange above the coldest temperature
    z = np.where(valid, mean / np.where(se > 0, se, 1.0), 0.0)
    names = ["E/N", "acc", "exchange", "q2"] + [f"P(q) bin {b}" for b in range(len(QBINS) - 1)]
    report = {name: np.round(z[i], 2).tolist() for i, name in enumerate(names)}
    print(variant, "paired z-scores per temperature:", report)
    print("engine E/N per T:", np.round(obs_o[:, 0].mean(axis=0), 4).tolist())
    print("reference E/N per T:", np.round(obs_r[:, 0].mean(axis=0), 4).tolist())
    zs = np.abs(z[valid])
    n_out = int(np.sum(zs > 2.0))
    print(f"{variant}: {zs.size} z-scores, {n_out} outside 2 sigma ({100.0 * n_out / zs.size:.1f} %), "
          f"largest |z| {zs.max():.2f}")
    assert np.all(zs < 4.0), report
    assert n_out <= 0.10 * zs.size, report
