"""Host parts of the GPU P(q) analysis: configs.bin and energy_accept.txt
reading, run discovery, and the jackknife / file format of
parisi_overlap.dat (analysis_pt.cpp:1418-1480), on synthetic files."""
import os

import numpy as np

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
