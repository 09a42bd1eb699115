"""Host parts of the GPU overlap analyses: configs.bin and energy_accept.txt
reading, run discovery, the jackknife / file format of parisi_overlap.dat
(analysis_pt.cpp:1418-1480), and every file analysis_pt derives from the
P(q), IFO and experimental-IFO histograms (distributions, moments, glass
observables, per-sample <x^2>) checked byte for byte against the reference
analysis_pt, on synthetic files."""
import math
import os
import subprocess

import numpy as np
import pytest

from cuda_pspin_b200 import analysis as A


def _fake_run(d, N, NT, nrep, nsnap, rng, label):
    os.makedirs(d, exist_ok=True)
    cfg = rng.normal(size=(nsnap, NT, nrep, N, 2))
    with open(os.path.join(d, "configs.bin"), "wb") as f:
        np.array([N, NT, nrep], np.int32).tofile(f)
        for s in range(nsnap):
            np.array([1000 + 10 * s], np.int32).tofile(f)
            cfg[s].astype(np.float64).tofile(f)
    with open(os.path.join(d, "energy_accept.txt"), "w") as f:
        f.write("# sweep\tTidx\tT\n")
        for s in range(3):
            for t in range(NT):
                f.write("%d\t%d\t%.8f\t-1.0\t0.5\n" % (s, t, 1.5 - 0.25 * t))
    return cfg


def test_reading_and_discovery(tmp_path):
    rng = np.random.default_rng(0)
    a = _fake_run(tmp_path / "data" / "PT_N6_NT3_NR2_S1", 6, 3, 2, 4, rng, 1)
    _fake_run(tmp_path / "data" / "PT_N6_NT3_NR2_S0", 6, 3, 2, 2, rng, 0)
    _fake_run(tmp_path / "data" / "PT_N7_NT3_NR2_S2", 7, 3, 2, 2, rng, 2)      # other N: skipped
    runs = A.find_runs(str(tmp_path / "data"), 6, 3, 2)
    assert [l for l, _ in runs] == [0, 1]
    got = A.read_configs(runs[1][1], 6, 3, 2)
    np.testing.assert_array_equal(got, a)
    np.testing.assert_array_equal(A.temperatures(runs[1][1], 3), [1.5, 1.25, 1.0])


def test_jackknife_file(tmp_path):
    rng = np.random.default_rng(1)
    S, NT, nbins = 5, 2, 10
    h = rng.random((S, NT, nbins))
    path = str(tmp_path / "p.dat")
    A.write_parisi_overlap(path, h, [1.2, 0.4], 8, NT, 3, nbins)
    lines = open(path).read().splitlines()
    assert lines[1] == "# N=8 NT=2 nrep=3 nbins=10 nsamples=5"
    rows = np.array([[float(x) for x in l.split()] for l in lines if l and not l.startswith("#")])
    assert rows.shape == (NT * nbins, 4)
    mean = h.mean(axis=0)
    loo = (h.sum(axis=0)[None] - h) / (S - 1)
    err = np.sqrt((S - 1) / S * ((loo - mean[None]) ** 2).sum(axis=0))
    np.testing.assert_allclose(rows[:, 1], mean.ravel(), rtol=1e-8)
    np.testing.assert_allclose(rows[:, 2], err.ravel(), rtol=1e-8)
    np.testing.assert_allclose(rows[:nbins, 0], -1 + (np.arange(nbins) + 0.5) * 0.2, atol=1e-12)
    assert set(rows[:nbins, 3]) == {1.2} and set(rows[nbins:, 3]) == {0.4}


# ---- IFO / experimental IFO: restatement of the reference's FP64 order ------
def _intensity(x, k):
    return x[k, 0] * x[k, 0] + x[k, 1] * x[k, 1]


def _ifo_restated(cfg, nbins):
    """Plain-Python (round-to-nearest doubles, no contraction) restatement of
    analysis_pt.cpp:1547-1607 (IFO) and :1745-1793 (experimental IFO) in the
    operation order pspin_ifo_counts uses: densities [NT, nbins] of each."""
    nsnap, NT, nrep, N, _ = cfg.shape
    cmin, dc = -1.0, 2.0 / nbins
    ifo, ex = np.zeros((NT, nbins)), np.zeros((NT, nbins))

    def add(cnt, num, den):
        if den <= 0:
            return 0
        cnt[min(max(int((num / den - cmin) / dc), 0), nbins - 1)] += 1
        return 1
    for t in range(NT):
        mean = []
        for r in range(nrep):
            row = []
            for k in range(N):
                s = 0.0
                for sn in range(nsnap):
                    s = s + _intensity(cfg[sn, t, r], k)
                row.append(s / nsnap)
            mean.append(row)
        cnt, n = [0] * nbins, 0
        for sn in range(nsnap):
            d = [[_intensity(cfg[sn, t, r], k) - mean[r][k] for k in range(N)] for r in range(nrep)]
            n2 = []
            for r in range(nrep):
                s = 0.0
                for k in range(N):
                    s = s + d[r][k] * d[r][k]
                n2.append(s)
            for a in range(nrep):
                for b in range(a + 1, nrep):
                    num = 0.0
                    for k in range(N):
                        num = num + d[a][k] * d[b][k]
                    n += add(cnt, num, math.sqrt(n2[a] * n2[b]))
        if n:
            ifo[t] = np.array(cnt) / (n * dc)
        g = []
        for k in range(N):
            s = 0.0
            for r in range(nrep):
                s = s + mean[r][k]
            g.append(s / nrep)
        d = [[mean[r][k] - g[k] for k in range(N)] for r in range(nrep)]
        cnt, n = [0] * nbins, 0
        for a in range(nrep):
            for b in range(a + 1, nrep):
                na = nb = num = 0.0
                for k in range(N):
                    na = na + d[a][k] * d[a][k]
                    nb = nb + d[b][k] * d[b][k]
                    num = num + d[a][k] * d[b][k]
                n += add(cnt, num, math.sqrt(na * nb))
        if n:
            ex[t] = np.array(cnt) / (n * dc)
    return ifo, ex


REF_ANALYSIS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                            "analysis_pt")


def _pq_restated(cfg, nbins):
    """P(q) densities [NT, nbins] in pspin_overlap_counts' operation order
    (analysis_pt.cpp:1385-1424)."""
    nsnap, NT, nrep, N, _ = cfg.shape
    qmin, dq = -1.0, 2.0 / nbins
    out = np.zeros((NT, nbins))
    for t in range(NT):
        cnt = [0] * nbins
        for sn in range(nsnap):
            for a in range(nrep):
                for b in range(a + 1, nrep):
                    s = 0.0
                    for k in range(N):
                        x, y = cfg[sn, t, a, k], cfg[sn, t, b, k]
                        s = s + (x[0] * y[0] + x[1] * y[1])
                    cnt[min(max(int((s / N - qmin) / dq), 0), nbins - 1)] += 1
        out[t] = np.array(cnt) / (nsnap * nrep * (nrep - 1) // 2 * dq)
    return out


@pytest.mark.skipif(not os.path.exists(REF_ANALYSIS), reason="reference analysis_pt not built")
@pytest.mark.parametrize("S", [4, 1])
def test_overlap_files_match_analysis_pt(tmp_path, S):
    """The operation order of pspin_overlap_counts and pspin_ifo_counts,
    restated on the CPU, and analysis.write_all (distributions, moments,
    glass observables, per-sample <x^2>) give the same twelve files as the
    reference analysis_pt on synthetic runs, byte for byte: including an
    overlap of exactly 1 (two identical replicas: the last bin), a replica
    with no fluctuation (zero norm: skipped and not counted) and, with one
    sample, the reference's -nan jackknife errors."""
    N, NT, nrep, nsnap, nbins = 6, 3, 3, 5, 20
    rng = np.random.default_rng(5 + S)
    cfgs = []
    for s in range(S):
        d = tmp_path / "data" / f"PT_N{N}_a0.5_Rinf_a00.5_NT{NT}_NR{nrep}_S{s}"
        cfg = _fake_run(str(d), N, NT, nrep, nsnap, rng, s)
        if s == S - 1:
            cfg[:, 0, 2] = cfg[:, 0, 1]
            cfg[:, 1, 0] = cfg[0, 1, 0]
            with open(d / "configs.bin", "wb") as f:
                np.array([N, NT, nrep], np.int32).tofile(f)
                for k in range(nsnap):
                    np.array([1000 + 10 * k], np.int32).tofile(f)
                    cfg[k].tofile(f)
        with open(d / "energy_accept.txt", "w") as f:           # nrep (E, acc) columns
            f.write("# sweep\tTidx\tT" + "".join(f"\tE{r}/N\tacc{r}" for r in range(nrep)) + "\n")
            for sw in range(3):
                for t in range(NT):
                    f.write("%d\t%d\t%.8f" % (sw, t, 1.5 - 0.25 * t) + "\t-1.00000000\t0.50000" * nrep + "\n")
        with open(d / "exchanges.txt", "w") as f:
            f.write("# sweep\tTidx\tT_high\tT_low\tn_acc\tn_prop\trate\n")
            for sw in range(3):
                for t in range(NT - 1):
                    f.write("%d\t%d\t%.8f\t%.8f\t1\t2\t0.50000\n" % (sw, t, 1.5 - 0.25 * t, 1.25 - 0.25 * t))
        cfgs.append(cfg)
    p = subprocess.run([REF_ANALYSIS, "-N", str(N), "-NT", str(NT), "-nrep", str(nrep), "-nbins", str(nbins)],
                       cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-1000:]
    ifo = [_ifo_restated(c, nbins) for c in cfgs]
    hists = {"parisi": np.stack([_pq_restated(c, nbins) for c in cfgs]),
             "ifo": np.stack([r[0] for r in ifo]), "exp_ifo": np.stack([r[1] for r in ifo])}
    temps = A.temperatures(str(tmp_path / "data" / f"PT_N{N}_a0.5_Rinf_a00.5_NT{NT}_NR{nrep}_S0"), NT)
    paths = A.write_all(str(tmp_path / "ours"), hists, temps, N, NT, nrep, nbins)
    assert len(paths) == 12
    refdir = [r for r, _, fs in os.walk(tmp_path / "analysis") if "parisi_overlap.dat" in fs]
    assert len(refdir) == 1
    for path in paths:
        ref = os.path.join(refdir[0], os.path.basename(path))
        assert open(path).read() == open(ref).read(), os.path.basename(path)
    if S == 1:
        assert "-nan" in open(paths[1]).read()


@pytest.mark.skipif(not os.path.exists(REF_ANALYSIS), reason="reference analysis_pt not built")
def test_decorrelation_time_matches_analysis_pt(tmp_path):
    """tau_E (pspin_tau_e on the host, analysis.write_tau_e) against the
    reference analysis_pt's decorrelation_time.dat, byte for byte, on
    synthetic runs whose energy series are AR(1) processes of different
    correlation per temperature (crossings of 1/e with and without
    interpolation, a series that never crosses, a constant one)."""
    N, NT, nrep, nsnap = 6, 4, 3, 2
    rng = np.random.default_rng(11)
    M = 80
    for s in range(3):
        d = tmp_path / "data" / f"PT_N{N}_a0.5_Rinf_a00.5_NT{NT}_NR{nrep}_S{s}"
        _fake_run(str(d), N, NT, nrep, nsnap, rng, s)
        series = np.zeros((NT, M, nrep))
        for t, phi in enumerate((0.2, 0.8, 0.995, None)):
            if phi is None:
                series[t] = -1.25
                continue
            x = rng.normal(size=nrep)
            for i in range(M):
                x = phi * x + rng.normal(size=nrep)
                series[t, i] = -1.0 + 0.01 * x
        with open(d / "energy_accept.txt", "w") as f:
            f.write("# sweep\tTidx\tT" + "".join(f"\tE{r}/N\tacc{r}" for r in range(nrep)) + "\n")
            for i in range(M):
                for t in range(NT):
                    f.write("%d\t%d\t%.8f" % (10 * (i + 1), t, 1.5 - 0.25 * t) +
                            "".join("\t%.8f\t0.50000" % series[t, i, r] for r in range(nrep)) + "\n")
        with open(d / "exchanges.txt", "w") as f:
            f.write("# sweep\tTidx\tT_high\tT_low\tn_acc\tn_prop\trate\n")
            for i in range(M):
                for t in range(NT - 1):
                    f.write("%d\t%d\t%.8f\t%.8f\t1\t2\t0.50000\n" % (10 * (i + 1), t, 1.5 - 0.25 * t,
                                                                   1.25 - 0.25 * t))
    p = subprocess.run([REF_ANALYSIS, "-N", str(N), "-NT", str(NT), "-nrep", str(nrep)],
                       cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-1000:]
    runs = A.find_runs(str(tmp_path / "data"), N, NT, nrep)
    temps = A.temperatures(runs[0][1], NT)
    os.makedirs(tmp_path / "ours")
    path = A.write_tau_e(str(tmp_path / "ours"), runs, NT, nrep, temps)
    refdir = [r for r, _, fs in os.walk(tmp_path / "analysis") if "decorrelation_time.dat" in fs]
    assert len(refdir) == 1
    ours = open(path).read()
    assert ours == open(os.path.join(refdir[0], "decorrelation_time.dat")).read()
    vals = [float(l.split()[1]) for l in ours.splitlines() if not l.startswith("#")]
    assert vals[0] > 0 and vals[2] > vals[1] > vals[0] and vals[3] == 0.0
