"""Parisi overlap distribution P(q) of a set of PT runs, computed on the GPU.

Reads the runs' configs.bin files (the engine's or the reference's drivers
write the same format), histograms q_ab = Re sum_k a_k^a conj(a_k^b) / N over
every saved configuration and replica pair at each temperature with
`pspin_overlap_counts` (binned exactly as the reference bins), normalises
each sample's histogram to a density and writes parisi_overlap.dat with the
sample mean and jackknife error in the reference's format
(analysis_pt.cpp:1337-1480):

    python -m cuda_pspin_b200.analysis -N 12 -NT 4 -nrep 2 [-nbins 100] [--data data] [--out analysis_gpu]
"""
from __future__ import annotations

import argparse
import os
import re
import sys

import numpy as np

from . import _check, _ptr, load_library


def find_runs(data_dir: str, N: int, NT: int, nrep: int) -> list[tuple[int, str]]:
    """(label, dir) of every run under data_dir whose configs.bin header is (N, NT, nrep), by label."""
    runs = []
    for name in os.listdir(data_dir):
        d = os.path.join(data_dir, name)
        m = re.search(r"_S(-?\d+)$", name)
        f = os.path.join(d, "configs.bin")
        if not m or not os.path.isfile(f):
            continue
        hdr = np.fromfile(f, dtype=np.int32, count=3)
        if tuple(hdr) == (N, NT, nrep):
            runs.append((int(m.group(1)), d))
    return sorted(runs)


def read_configs(d: str, N: int, NT: int, nrep: int) -> np.ndarray:
    """configs.bin body as [nsnap, NT, nrep, N, 2] float64 (sweep numbers dropped)."""
    raw = np.fromfile(os.path.join(d, "configs.bin"), dtype=np.uint8)[12:]
    rec = 4 + NT * nrep * 2 * N * 8
    nsnap = len(raw) // rec
    body = raw[:nsnap * rec].reshape(nsnap, rec)[:, 4:]
    return np.ascontiguousarray(body).view(np.float64).reshape(nsnap, NT, nrep, N, 2)


def temperatures(d: str, NT: int) -> np.ndarray:
    """T of each temperature index, from energy_accept.txt (its T column as written)."""
    T = np.full(NT, np.nan)
    with open(os.path.join(d, "energy_accept.txt")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            tok = line.split()
            t = int(tok[1])
            if 0 <= t < NT and np.isnan(T[t]):
                T[t] = float(tok[2])
            if not np.isnan(T).any():
                break
    return T


def overlap_histograms(cfg: np.ndarray, nbins: int = 100, qmin: float = -1.0, qmax: float = 1.0) -> np.ndarray:
    """Densities [NT, nbins] of one sample: counts / (n_overlaps dq) as the reference normalises."""
    nsnap, NT, nrep, N, _ = cfg.shape
    counts = np.zeros((NT, nbins), np.int64)
    c = np.ascontiguousarray(cfg, np.float64)
    _check(load_library().pspin_overlap_counts(N, NT, nrep, nsnap, _ptr(c), nbins, qmin, qmax, _ptr(counts)))
    n_overlaps = nsnap * nrep * (nrep - 1) // 2
    dq = (qmax - qmin) / nbins
    return counts / (n_overlaps * dq) if n_overlaps > 0 else counts.astype(np.float64)


def write_parisi_overlap(path: str, hists: np.ndarray, temps, N: int, NT: int, nrep: int, nbins: int,
                         qmin: float = -1.0, qmax: float = 1.0) -> None:
    """hists [nsamples, NT, nbins]; the sample mean and jackknife error per bin."""
    S = hists.shape[0]
    dq = (qmax - qmin) / nbins
    with open(path, "w") as f:
        f.write("# Parisi overlap distribution P(q)\n")
        f.write(f"# N={N} NT={NT} nrep={nrep} nbins={nbins} nsamples={S}\n")
        f.write("# q = Re[ (1/N) sum_i a_i^alpha * conj(a_i^beta) ]\n")
        f.write("# Columns: q_center  P(q)  Error_jk  Temperature\n")
        f.write("# NT blocks separated by blank lines\n")
        for ti in range(hists.shape[1]):
            f.write("\n")
            for b in range(nbins):
                qc = qmin + (b + 0.5) * dq
                col = [float(hists[s, ti, b]) for s in range(S)]
                fP = 0.0
                for v in col:
                    fP += v
                fP /= S
                jP = 0.0
                for j in range(S):
                    lP = 0.0
                    for s in range(S):
                        if s != j:
                            lP += col[s]
                    lP /= (S - 1)
                    jP += (lP - fP) * (lP - fP)
                jP = np.sqrt((S - 1.0) / S * jP)
                f.write("%.12f\t%.8e\t%.8e\t%.8f\n" % (qc, fP, jP, temps[ti]))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-N", type=int, required=True)
    ap.add_argument("-NT", type=int, required=True)
    ap.add_argument("-nrep", type=int, required=True)
    ap.add_argument("-nbins", type=int, default=100)
    ap.add_argument("--data", default="data")
    ap.add_argument("--out", default="analysis_gpu")
    a = ap.parse_args(argv)
    runs = find_runs(a.data, a.N, a.NT, a.nrep)
    if not runs:
        print("no runs with N=%d NT=%d nrep=%d under %s" % (a.N, a.NT, a.nrep, a.data), file=sys.stderr)
        return 1
    hists = np.stack([overlap_histograms(read_configs(d, a.N, a.NT, a.nrep), a.nbins) for _, d in runs])
    temps = temperatures(runs[0][1], a.NT)
    os.makedirs(a.out, exist_ok=True)
    path = os.path.join(a.out, "parisi_overlap.dat")
    write_parisi_overlap(path, hists, temps, a.N, a.NT, a.nrep, a.nbins)
    print("%d samples, written %s" % (len(runs), path))
    return 0


if __name__ == "__main__":
    sys.exit(main())
