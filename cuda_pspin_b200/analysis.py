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
With --deeper, as analysis_pt --deeper does: P(|a|^2) and the inverse
participation ratios, the phase overlap and, for runs with quartets.txt,
the link overlap and the q-q_link scatter (`pspin_deeper_counts`,
analysis_pt.cpp:1871-2290), and the multi-overlap scatter files
(`pspin_multi_overlap`, :3468-3643).  Always: the energy decorrelation time
tau_E (decorrelation_time.dat, :2694-2790; `pspin_tau_e` on the host).
Each sample's histogram is normalised to a density and the files hold the
sample mean and jackknife error in the reference's format; from the same
histograms, as analysis_pt does for each distribution (tags parisi, ifo,
exp_ifo): {tag}_moments.dat (mean, variance, skewness, excess kurtosis with
jackknife errors, analysis_pt.cpp:61-126), {tag}_glass_observables.dat (chi
= N<x^2>, Binder g4, non-self-averaging A) and {tag}_sample_x2.dat
(:209-305).  The host arithmetic follows the reference's operation order in
IEEE doubles, so the printed numbers are the reference's (a single sample
gives its -nan jackknife errors):

    python -m cuda_pspin_b200.analysis -N 12 -NT 4 -nrep 2 [-nbins 100] [--deeper] [--data data] [--out analysis_gpu]
"""
from __future__ import annotations

import argparse
import ctypes
import math
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


# ---- host arithmetic in the reference's order (IEEE doubles, x86 results) ---
def _div(a, b):
    """a / b with C's result for b == 0 (inf, or the negative default NaN)."""
    if b == 0:
        with np.errstate(all="ignore"):
            return float(np.float64(a) / np.float64(b))
    return a / b


def _e(x) -> str:
    """printf("%.8e") as glibc prints it (a NaN with its sign)."""
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    return "%.8e" % x


def _mean_rows(h: np.ndarray, skip: int = -1) -> np.ndarray:
    """Per-bin sum over the samples s != skip in sample order, divided by
    their count: h [S, nbins] (vectorised over bins only)."""
    acc = np.zeros(h.shape[1])
    n = 0
    for s in range(h.shape[0]):
        if s != skip:
            acc = acc + h[s]
            n += 1
    with np.errstate(all="ignore"):
        return acc / np.float64(n)


def write_parisi_overlap(path: str, hists: np.ndarray, temps, N: int, NT: int, nrep: int, nbins: int,
                         qmin: float = -1.0, qmax: float = 1.0, header=PARISI_HEADER) -> None:
    """hists [nsamples, NT, nbins]; the sample mean and jackknife error per bin
    under the given header lines (the P(q), IFO and experimental-IFO files
    share this layout; analysis_pt.cpp:1452-1477)."""
    hists = np.asarray(hists, np.float64)
    S = hists.shape[0]
    dq = (qmax - qmin) / nbins
    with open(path, "w") as f:
        for line in header:
            f.write(line.format(N=N, NT=NT, nrep=nrep, nbins=nbins, S=S) + "\n")
        for ti in range(hists.shape[1]):
            f.write("\n")
            h = hists[:, ti, :]
            fP = _mean_rows(h)
            jP = np.zeros(nbins)
            for j in range(S):
                lP = _mean_rows(h, j)
                jP = jP + (lP - fP) * (lP - fP)
            with np.errstate(all="ignore"):
                jP = np.sqrt((S - 1.0) / S * jP)
            for b in range(nbins):
                qc = qmin + (b + 0.5) * dq
                f.write("%.12f\t%s\t%s\t%.8f\n" % (qc, _e(float(fP[b])), _e(float(jP[b])), temps[ti]))


def hist_moments(h, nbins: int, xmin: float, dx: float):
    """Mean, variance, skewness, excess kurtosis of a density histogram
    (analysis_pt.cpp:61-81)."""
    h = [float(v) for v in h]
    mu = 0.0
    for b in range(nbins):
        xc = xmin + (b + 0.5) * dx
        mu += xc * h[b] * dx
    var = skew = kurt = 0.0
    for b in range(nbins):
        xc = xmin + (b + 0.5) * dx
        d = xc - mu
        d2 = d * d
        var += d2 * h[b] * dx
        skew += d2 * d * h[b] * dx
        kurt += d2 * d2 * h[b] * dx
    if var > 0:
        skew = _div(skew, var * math.sqrt(var))
        kurt = _div(kurt, var * var) - 3.0
    return mu, var, skew, kurt


def write_moments(path: str, header: str, hists: np.ndarray, temps, nbins: int, xmin: float = -1.0,
                  dx: float | None = None) -> None:
    """{tag}_moments.dat: moments of the sample-mean histogram per
    temperature with jackknife errors (analysis_pt.cpp:86-126)."""
    hists = np.asarray(hists, np.float64)
    S, NT = hists.shape[0], hists.shape[1]
    dx = 2.0 / nbins if dx is None else dx
    f = math.sqrt((S - 1.0) / S)
    with open(path, "w") as out:
        out.write("# %s\n" % header)
        out.write("# Columns: T  mean  mean_err  var  var_err  skew  skew_err  kurt  kurt_err\n")
        for ti in range(NT):
            h = hists[:, ti, :]
            full = hist_moments(_mean_rows(h), nbins, xmin, dx)
            jk = [0.0, 0.0, 0.0, 0.0]
            for j in range(S):
                loo = hist_moments(_mean_rows(h, j), nbins, xmin, dx)
                for m in range(4):
                    jk[m] += (loo[m] - full[m]) * (loo[m] - full[m])
            cols = []
            for m in range(4):
                cols += [full[m], f * math.sqrt(jk[m])]
            out.write("%.8f\t" % temps[ti] + "\t".join(_e(c) for c in cols) + "\n")


def write_glass_observables(outdir: str, tag: str, hists: np.ndarray, temps, N: int, nbins: int,
                            xmin: float = -1.0, dx: float | None = None) -> None:
    """{tag}_glass_observables.dat (chi = N<x^2>, g4 = (3 - <x^4>/<x^2>^2)/2,
    A = Var_J[<x^2>]/<x^2>^2 with jackknife errors) and {tag}_sample_x2.dat
    (analysis_pt.cpp:209-305)."""
    hists = np.asarray(hists, np.float64)
    S, NT = hists.shape[0], hists.shape[1]
    dx = 2.0 / nbins if dx is None else dx
    x2 = [[0.0] * NT for _ in range(S)]
    x4 = [[0.0] * NT for _ in range(S)]
    for s in range(S):
        for ti in range(NT):
            m2 = m4 = 0.0
            for b in range(nbins):
                xc = xmin + (b + 0.5) * dx
                xc2 = xc * xc
                v = float(hists[s, ti, b])
                m2 += xc2 * v * dx
                m4 += xc2 * xc2 * v * dx
            x2[s][ti], x4[s][ti] = m2, m4
    f = math.sqrt((S - 1.0) / S)
    rows = []
    for ti in range(NT):
        x2f = x4f = 0.0
        for s in range(S):
            x2f += x2[s][ti]
            x4f += x4[s][ti]
        x2f = _div(x2f, S)
        x4f = _div(x4f, S)
        chi = N * x2f
        g4 = 0.5 * (3.0 - _div(x4f, x2f * x2f)) if x2f > 0 else 0.0
        x2v = 0.0
        for s in range(S):
            x2v += (x2[s][ti] - x2f) * (x2[s][ti] - x2f)
        x2v = _div(x2v, S)
        A = _div(x2v, x2f * x2f) if x2f > 0 else 0.0
        jc = jg = jA = 0.0
        for j in range(S):
            lx2 = lx4 = 0.0
            for s in range(S):
                if s != j:
                    lx2 += x2[s][ti]
                    lx4 += x4[s][ti]
            lx2 = _div(lx2, S - 1)
            lx4 = _div(lx4, S - 1)
            lchi = N * lx2
            lg4 = 0.5 * (3.0 - _div(lx4, lx2 * lx2)) if lx2 > 0 else 0.0
            jc += (lchi - chi) * (lchi - chi)
            jg += (lg4 - g4) * (lg4 - g4)
            lv = 0.0
            for s in range(S):
                if s != j:
                    lv += (x2[s][ti] - lx2) * (x2[s][ti] - lx2)
            lv = _div(lv, S - 1)
            lA = _div(lv, lx2 * lx2) if lx2 > 0 else 0.0
            jA += (lA - A) * (lA - A)
        rows.append((temps[ti], chi, f * math.sqrt(jc), g4, f * math.sqrt(jg), A, f * math.sqrt(jA)))
    with open(os.path.join(outdir, "%s_glass_observables.dat" % tag), "w") as out:
        out.write("# Glass observables from %s overlap\n" % tag)
        out.write("# chi = N*<x^2>,  g4 = 0.5*(3-<x^4>/<x^2>^2),  A = Var_J[<x^2>]/<x^2>^2\n")
        out.write("# Columns: T  chi  chi_err  g4  g4_err  A  A_err\n")
        for r in rows:
            out.write("%.8f\t" % r[0] + "\t".join(_e(c) for c in r[1:]) + "\n")
    with open(os.path.join(outdir, "%s_sample_x2.dat" % tag), "w") as out:
        out.write("# Per-sample <x^2> for %s\n" % tag)
        out.write("# Columns: T  sample_0  sample_1  ...  sample_{n-1}\n")
        for ti in range(NT):
            out.write("%.8f" % temps[ti] + "".join("\t" + _e(x2[s][ti]) for s in range(S)) + "\n")


def read_quartets(d: str) -> np.ndarray:
    """quartets.txt of a sparse run as [M, 5] int32 (i, j, k, l, ch); empty
    when the file is absent (analysis_pt.cpp:314-330)."""
    path = os.path.join(d, "quartets.txt")
    rows = []
    if os.path.isfile(path):
        with open(path) as f:
            for line in f:
                if line.startswith("#") or line.startswith("\n"):
                    continue
                tok = line.split()
                if len(tok) >= 7:
                    try:
                        rows.append([int(tok[1]), int(tok[2]), int(tok[3]), int(tok[4]), int(tok[5])])
                        float(tok[6])
                    except ValueError:
                        continue
    return np.array(rows, np.int32).reshape(-1, 5)


def energy_rows(d: str, NT: int, nrep: int) -> list[np.ndarray]:
    """energy_accept.txt's E/N columns per temperature index, rows in file
    order ([M_t, nrep] each; analysis_pt.cpp:501-565)."""
    out = [[] for _ in range(NT)]
    with open(os.path.join(d, "energy_accept.txt")) as f:
        for line in f:
            if line.startswith("#") or line.startswith("\n"):
                continue
            tok = line.split()
            if len(tok) < 3 + 2 * nrep:
                continue
            t = int(tok[1])
            if 0 <= t < NT:
                out[t].append([float(tok[3 + 2 * r]) for r in range(nrep)])
    return [np.array(r, np.float64).reshape(-1, nrep) for r in out]


def tau_e(rows: np.ndarray) -> float:
    """The reference's tau_E of one temperature (pspin_tau_e)."""
    r = np.ascontiguousarray(rows, np.float64)
    t = ctypes.c_double()
    if load_library().pspin_tau_e(int(r.shape[0]), int(r.shape[1]), _ptr(r), ctypes.byref(t)) != 0:
        raise ValueError("pspin_tau_e: bad arguments")
    return t.value


def write_tau_e(outdir: str, runs, NT: int, nrep: int, temps) -> str:
    """decorrelation_time.dat: tau_E per temperature, sample mean and
    jackknife error (analysis_pt.cpp:2755-2788)."""
    S = len(runs)
    tau = [[0.0] * NT for _ in range(S)]
    for s, (_, d) in enumerate(runs):
        rows = energy_rows(d, NT, nrep)
        for ti in range(NT):
            tau[s][ti] = tau_e(rows[ti])
    path = os.path.join(outdir, "decorrelation_time.dat")
    with open(path, "w") as f:
        f.write("# Energy decorrelation time tau_E (in save_freq units)\n")
        f.write("# T\ttau_E\ttau_E_err\n")
        for ti in range(NT):
            vals = [tau[s][ti] for s in range(S)]
            fm = 0.0
            for v in vals:
                fm += v
            fm = _div(fm, S)
            jk = 0.0
            for j in range(S):
                lv = 0.0
                for s in range(S):
                    if s != j:
                        lv += vals[s]
                lv = _div(lv, S - 1)
                jk += (lv - fm) * (lv - fm)
            jk = math.sqrt((S - 1.0) / S * jk) if S > 0 else float("nan")
            f.write("%.8f\t%s\t%s\n" % (temps[ti], _e(fm), _e(jk)))
    return path


NBINS_A2, A2_MAX = 100, 10.0
MARGINAL_HEADER = ["# Marginal distribution P(|a_k|^2 = I_k)", "# Columns: I_center  P(I)  Error_jk  Temperature"]
PHASE_HEADER = ["# Phase overlap distribution P(q_phi)", "# q_phi = (1/N_eff) sum_k cos(theta_k^a - theta_k^b)",
                "# Columns: q_phi_center  P(q_phi)  Error_jk  Temperature"]
LINK_HEADER = ["# Link overlap distribution P(q_link)",
               "# q_link = (1/M) sum_q t_q(a)*t_q(b),  t_q = Re[prod with channel]",
               "# Columns: q_link_center  P(q_link)  Error_jk  Temperature"]


def deeper_sample(cfg: np.ndarray, nbins: int, quarts: np.ndarray):
    """One sample's deeper-block results (analysis_pt.cpp:1871-2045):
    marginal, phase and link densities [NT, bins], Y2 and Y4 per temperature
    and the (q, q_link) scatter points per temperature, normalised in the
    reference's order."""
    nsnap, NT, nrep, N, _ = cfg.shape
    npairs = nrep * (nrep - 1) // 2
    M = int(quarts.shape[0])
    marg = np.zeros((NT, NBINS_A2), np.int64)
    phase = np.zeros((NT, nbins), np.int64)
    link = np.zeros((NT, nbins), np.int64)
    y = np.zeros((nsnap, NT, nrep, 3))
    sc = np.zeros((NT, nsnap, npairs, 2))
    c = np.ascontiguousarray(cfg, np.float64)
    q = np.ascontiguousarray(quarts, np.int32) if M else np.zeros((1, 5), np.int32)
    _check(load_library().pspin_deeper_counts(N, NT, nrep, nsnap, _ptr(c), nbins, NBINS_A2, A2_MAX, _ptr(q), M,
                                              _ptr(marg), _ptr(y), _ptr(phase), _ptr(link), _ptr(sc)))
    da2 = A2_MAX / NBINS_A2
    dq = 2.0 / nbins
    md, pd, ld = marg.astype(np.float64), phase.astype(np.float64), link.astype(np.float64)
    y2, y4, scat = [0.0] * NT, [0.0] * NT, []
    for t in range(NT):
        n_ipr, a2, a4 = 0, 0.0, 0.0
        for sn in range(nsnap):
            for r in range(nrep):
                if y[sn, t, r, 2] != 0.0:
                    a2 += float(y[sn, t, r, 0])
                    a4 += float(y[sn, t, r, 1])
                    n_ipr += 1
        if n_ipr * N > 0:
            md[t] = md[t] / (float(n_ipr * N) * da2)
        if n_ipr > 0:
            a2 /= n_ipr
            a4 /= n_ipr
        y2[t], y4[t] = a2, a4
        n_ph = nsnap * npairs
        if n_ph > 0:
            pd[t] = pd[t] / (n_ph * dq)
            if M:
                ld[t] = ld[t] / (n_ph * dq)
        scat.append(sc[t].reshape(-1, 2) if M else np.zeros((0, 2)))
    return md, pd, ld, np.array(y2), np.array(y4), scat


def _write_ipr(outdir: str, y2: np.ndarray, y4: np.ndarray, temps) -> list[str]:
    S, NT = y2.shape
    ff = math.sqrt((S - 1.0) / S)
    p1, p2 = os.path.join(outdir, "ipr.dat"), os.path.join(outdir, "ipr_sample.dat")
    with open(p1, "w") as f:
        f.write("# Inverse Participation Ratios\n")
        f.write("# Y2 = sum I_k^2 / (sum I_k)^2,  Y4 = sum I_k^4 / (sum I_k)^4\n")
        f.write("# 1/Y2 = effective number of participating modes\n")
        f.write("# Columns: T  Y2  Y2_err  Y4  Y4_err\n")
        for ti in range(NT):
            y2f = y4f = 0.0
            for s in range(S):
                y2f += float(y2[s, ti])
                y4f += float(y4[s, ti])
            y2f = _div(y2f, S)
            y4f = _div(y4f, S)
            j2 = j4 = 0.0
            for j in range(S):
                l2 = l4 = 0.0
                for s in range(S):
                    if s != j:
                        l2 += float(y2[s, ti])
                        l4 += float(y4[s, ti])
                l2 = _div(l2, S - 1)
                l4 = _div(l4, S - 1)
                j2 += (l2 - y2f) * (l2 - y2f)
                j4 += (l4 - y4f) * (l4 - y4f)
            f.write("%.8f\t%s\t%s\t%s\t%s\n" % (temps[ti], _e(y2f), _e(ff * math.sqrt(j2)), _e(y4f),
                                                   _e(ff * math.sqrt(j4))))
    with open(p2, "w") as f:
        f.write("# Per-sample Y2 values\n")
        f.write("# Columns: T  sample_0  sample_1  ... sample_{n-1}\n")
        for ti in range(NT):
            f.write("%.8f" % temps[ti] + "".join("\t" + _e(float(y2[s, ti])) for s in range(S)) + "\n")
    return [p1, p2]


def write_deeper(outdir: str, runs, N: int, NT: int, nrep: int, nbins: int, temps) -> list[str]:
    """Every file of analysis_pt's deeper overlap block (P(|a|^2), IPR, phase
    and link overlaps with their moments and glass observables, the
    q-q_link scatter) and the multi-overlap scatter files."""
    os.makedirs(outdir, exist_ok=True)
    marg, phase, link, y2, y4, scat, has_q = [], [], [], [], [], [], False
    multi = [[] for _ in range(NT)]
    lib = load_library()
    npairs = nrep * (nrep - 1) // 2
    for s, (_, d) in enumerate(runs):
        cfg = read_configs(d, N, NT, nrep)
        quarts = read_quartets(d)
        has_q = has_q or quarts.shape[0] > 0
        m, p, l, a, b, sc = deeper_sample(cfg, nbins, quarts)
        marg.append(m); phase.append(p); link.append(l); y2.append(a); y4.append(b); scat.append(sc)
        # multi-overlap: snapshots in sweep order, shuffled and cut to 512 when more
        nsnap = cfg.shape[0]
        nit = min(nsnap, 512)
        snaps = np.zeros((NT, max(nit, 1)), np.int32)
        for ti in range(NT):
            idx = np.arange(nsnap, dtype=np.int32)
            if nsnap > 512:
                _check_rc(lib.pspin_std_shuffle(nsnap, (42 + s * NT + ti) & 0xFFFFFFFF, _ptr(idx)))
            snaps[ti, :nit] = idx[:nit]
        if nit > 0:
            out = np.zeros((NT, npairs, nit, 3))
            c = np.ascontiguousarray(cfg, np.float64)
            _check(lib.pspin_multi_overlap(N, NT, nrep, nsnap, _ptr(c), _ptr(snaps), nit, _ptr(out)))
            for ti in range(NT):
                multi[ti].append(out[ti].reshape(-1, 3))
    paths = []
    da2 = A2_MAX / NBINS_A2
    path = os.path.join(outdir, "marginal_a2.dat")
    write_parisi_overlap(path, np.stack(marg), temps, N, NT, nrep, NBINS_A2, 0.0, A2_MAX, header=MARGINAL_HEADER)
    paths.append(path)
    paths += _write_ipr(outdir, np.stack(y2), np.stack(y4), temps)
    for tag, hists, header, mheader in (("phase", phase, PHASE_HEADER, "Moments of P(q_phi)"),
                                        ("link", link, LINK_HEADER, "Moments of P(q_link)")):
        if tag == "link" and not has_q:
            continue
        h = np.stack(hists)
        path = os.path.join(outdir, "%s_overlap.dat" % tag)
        write_parisi_overlap(path, h, temps, N, NT, nrep, nbins, header=header)
        write_moments(os.path.join(outdir, "%s_moments.dat" % tag), mheader, h, temps, nbins)
        write_glass_observables(outdir, tag, h, temps, N, nbins)
        paths += [path, os.path.join(outdir, "%s_moments.dat" % tag),
                  os.path.join(outdir, "%s_glass_observables.dat" % tag),
                  os.path.join(outdir, "%s_sample_x2.dat" % tag)]
    if has_q:
        counts = np.array([sum(sc[ti].shape[0] for sc in scat) for ti in range(NT)], np.int64)
        pts = np.ascontiguousarray(np.concatenate([np.concatenate([sc[ti] for sc in scat]) for ti in range(NT)]),
                                   np.float64).reshape(-1, 2)
        kept = np.zeros_like(pts)
        kc = np.zeros(NT, np.int64)
        _check_rc(lib.pspin_fy_downsample(NT, _ptr(counts), 2, _ptr(pts), 2000, 42, _ptr(kept), _ptr(kc)))
        path = os.path.join(outdir, "scatter_q_qlink.dat")
        with open(path, "w") as f:
            f.write("# Scatter: Parisi overlap q vs Link overlap q_link\n")
            f.write("# Columns: q_parisi  q_link  Temperature\n")
            f.write("# (downsampled to max %d points per temperature)\n" % 2000)
            off = 0
            for ti in range(NT):
                f.write("\n")
                for p_ in kept[off:off + kc[ti]]:
                    f.write("%s\t%s\t%.8f\n" % (_e(float(p_[0])), _e(float(p_[1])), temps[ti]))
                off += kc[ti]
        paths.append(path)
    for ti in range(NT):
        if not multi[ti]:
            continue
        pts = np.ascontiguousarray(np.concatenate(multi[ti]), np.float64)
        kept = np.zeros((5000, 3))
        nk = ctypes.c_longlong()
        _check_rc(lib.pspin_reservoir_sample(pts.shape[0], 3, _ptr(pts), 5000, (42 + ti) & 0xFFFFFFFF, _ptr(kept),
                                             ctypes.byref(nk)))
        if nk.value == 0:
            continue
        path = os.path.join(outdir, "multi_overlap_T%.4f.dat" % temps[ti])
        with open(path, "w") as f:
            f.write("# Multi-overlap scatter at T=%.6f\n" % temps[ti])
            f.write("# q_parisi\tq_phase\tIFO\n")
            for p_ in kept[:nk.value]:
                f.write("%s\t%s\t%s\n" % (_e(float(p_[0])), _e(float(p_[1])), _e(float(p_[2]))))
        paths.append(path)
    return paths


def _check_rc(rc: int) -> None:
    if rc != 0:
        raise ValueError("bad arguments to a sampling helper")


# the three distributions: file stem / tag, moments header, distribution header
DISTRIBUTIONS = (("parisi", "Moments of P(q)", PARISI_HEADER),
                 ("ifo", "Moments of P(C) [IFO]", IFO_HEADER),
                 ("exp_ifo", "Moments of P(C) [exp-IFO]", EXP_IFO_HEADER))


def write_all(outdir: str, hists: dict, temps, N: int, NT: int, nrep: int, nbins: int) -> list[str]:
    """Every file analysis_pt writes from the overlap histograms, for the tags
    in hists ({tag: [nsamples, NT, nbins] densities}); returns the paths."""
    os.makedirs(outdir, exist_ok=True)
    paths = []
    for tag, mheader, header in DISTRIBUTIONS:
        if tag not in hists:
            continue
        name = "parisi_overlap.dat" if tag == "parisi" else "%s_overlap.dat" % tag
        write_parisi_overlap(os.path.join(outdir, name), hists[tag], temps, N, NT, nrep, nbins, header=header)
        write_moments(os.path.join(outdir, "%s_moments.dat" % tag), mheader, hists[tag], temps, nbins)
        write_glass_observables(outdir, tag, hists[tag], temps, N, nbins)
        paths += [name, "%s_moments.dat" % tag, "%s_glass_observables.dat" % tag, "%s_sample_x2.dat" % tag]
    return [os.path.join(outdir, p) for p in paths]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-N", type=int, required=True)
    ap.add_argument("-NT", type=int, required=True)
    ap.add_argument("-nrep", type=int, required=True)
    ap.add_argument("-nbins", type=int, default=100)
    ap.add_argument("--data", default="data")
    ap.add_argument("--out", default="analysis_gpu")
    ap.add_argument("--deeper", action="store_true", help="also the deeper block and the multi-overlap scatter")
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
    paths = write_all(a.out, {"parisi": np.stack(hists), "ifo": np.stack(ifo), "exp_ifo": np.stack(exp_ifo)},
                      temps, a.N, a.NT, a.nrep, a.nbins)
    paths.append(write_tau_e(a.out, runs, a.NT, a.nrep, temps))
    if a.deeper:
        paths += write_deeper(a.out, runs, a.N, a.NT, a.nrep, a.nbins, temps)
    for path in paths:
        print("%d samples, written %s" % (len(runs), path))
    return 0


if __name__ == "__main__":
    sys.exit(main())
