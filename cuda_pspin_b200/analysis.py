"""Overlap distributions of a set of PT runs, computed on the GPU.

Reads the runs' configs.bin files (the engine's or the reference's drivers
write the same format) and histograms, at each temperature and binned
exactly as the reference bins:
  * the Parisi overlap q_ab = Re sum_k a_k^a conj(a_k^b) / N over every saved
    configuration and replica pair (`pspin_overlap_counts`;
    analysis_pt.cpp:1337-1480 -> parisi_overlap.dat);
  * the intensity fluctuation overlap C_ab of I_k = |a_k|^2 about each
    replica's time average, per configuration and pair, and the
    experimental IFO of the time-averaged spectra, once per pair
    (`pspin_ifo_counts`; analysis_pt.cpp:1498-1663 -> ifo_overlap.dat,
    :1679-1850 -> exp_ifo_overlap.dat).
Each sample's histogram is normalised to a density and the files hold the
sample mean and jackknife error in the reference's format:

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


def ifo_histograms(cfg: np.ndarray, nbins: int = 100, cmin: float = -1.0,
                   cmax: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """IFO and experimental-IFO densities [NT, nbins] of one sample: counts /
    (overlaps counted * dC), zero where none was counted, as the reference
    normalises."""
    nsnap, NT, nrep, N, _ = cfg.shape
    ic, inn = np.zeros((NT, nbins), np.int64), np.zeros(NT, np.int64)
    ec, en = np.zeros((NT, nbins), np.int64), np.zeros(NT, np.int64)
    c = np.ascontiguousarray(cfg, np.float64)
    _check(load_library().pspin_ifo_counts(N, NT, nrep, nsnap, _ptr(c), nbins, cmin, cmax, _ptr(ic), _ptr(inn),
                                           _ptr(ec), _ptr(en)))
    dc = (cmax - cmin) / nbins

    def dens(counts, n):
        out = counts.astype(np.float64)
        for t in range(NT):
            if n[t] > 0:
                out[t] /= (n[t] * dc)
        return out
    return dens(ic, inn), dens(ec, en)


PARISI_HEADER = ["# Parisi overlap distribution P(q)", "# N={N} NT={NT} nrep={nrep} nbins={nbins} nsamples={S}",
                 "# q = Re[ (1/N) sum_i a_i^alpha * conj(a_i^beta) ]", "# Columns: q_center  P(q)  Error_jk  Temperature",
                 "# NT blocks separated by blank lines"]
IFO_HEADER = ["# Intensity Fluctuation Overlap (IFO) distribution P(C)",
              "# N={N} NT={NT} nrep={nrep} nbins={nbins} nsamples={S}",
              "# C^{{ab}} = sum_k delta_k^a delta_k^b / sqrt(sum_k (delta_k^a)^2 * sum_k (delta_k^b)^2)",
              "# delta_k^r = I_k^r - <I_k^r>_sweeps,  I_k = |a_k|^2", "# Columns: C_center  P(C)  Error_jk  Temperature",
              "# NT blocks separated by blank lines"]
EXP_IFO_HEADER = ["# Experimental IFO distribution P(C)", "# N={N} NT={NT} nrep={nrep} nbins={nbins} nsamples={S}",
                  "# delta_k^r = <I_k>_r - <<I_k>>,  <<I_k>> = (1/R) sum_r <I_k>_r",
                  "# C^{{ab}} = sum_k d_k^a d_k^b / sqrt(sum_k (d_k^a)^2 * sum_k (d_k^b)^2)",
                  "# Columns: C_center  P(C)  Error_jk  Temperature", "# NT blocks separated by blank lines"]


def write_parisi_overlap(path: str, hists: np.ndarray, temps, N: int, NT: int, nrep: int, nbins: int,
                         qmin: float = -1.0, qmax: float = 1.0, header=PARISI_HEADER) -> None:
    """hists [nsamples, NT, nbins]; the sample mean and jackknife error per bin
    under the given header lines (the P(q), IFO and experimental-IFO files
    share this layout)."""
    S = hists.shape[0]
    dq = (qmax - qmin) / nbins
    with open(path, "w") as f:
        for line in header:
            f.write(line.format(N=N, NT=NT, nrep=nrep, nbins=nbins, S=S) + "\n")
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
    hists, ifo, exp_ifo = [], [], []
    for _, d in runs:
        cfg = read_configs(d, a.N, a.NT, a.nrep)
        hists.append(overlap_histograms(cfg, a.nbins))
        i, e = ifo_histograms(cfg, a.nbins)
        ifo.append(i)
        exp_ifo.append(e)
    temps = temperatures(runs[0][1], a.NT)
    os.makedirs(a.out, exist_ok=True)
    for name, h, header in (("parisi_overlap.dat", hists, PARISI_HEADER), ("ifo_overlap.dat", ifo, IFO_HEADER),
                            ("exp_ifo_overlap.dat", exp_ifo, EXP_IFO_HEADER)):
        path = os.path.join(a.out, name)
        write_parisi_overlap(path, np.stack(h), temps, a.N, a.NT, a.nrep, a.nbins, header=header)
        print("%d samples, written %s" % (len(runs), path))
    return 0


if __name__ == "__main__":
    sys.exit(main())
