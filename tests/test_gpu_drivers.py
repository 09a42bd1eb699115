"""The drop-in drivers against the reference's own programs.

pspin_pt / pspin_pt_sparse / pspin_mc take the reference's flags and write
its files.  Each is run next to the reference's binary (rebuilt for sm_100a
from its sources into oracle/_ref/) with the same flags in separate working
directories:
  * files fixed by the disorder and the flags (params.txt, temperatures.txt,
    frequencies.txt, quartets.txt, the time.txt header) are byte-identical;
  * files with sampled values (energy_accept.txt, exchanges.txt,
    energy_split.txt, configs.bin) have the same headers, rows, columns and
    sizes;
  * the reference's analysis_pt reads the engine's output and completes.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cuda_pspin_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def run(cmd, cwd):
    p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p


def the_dir(base):
    data = os.path.join(base, "data")
    d = [x for x in os.listdir(data)]
    assert len(d) == 1, d
    return os.path.join(data, d[0])


def table(path):
    lines = open(path).read().splitlines()
    rows = [ln.split("\t") for ln in lines[1:]]
    return lines[0], rows


PT_FLAGS = ["-N", "12", "-Tmax", "1.6", "-Tmin", "0.2", "-NT", "4", "-log_temp", "-nrep", "2", "-iter", "64",
            "-pt_freq", "1", "-save_freq", "8", "-seed", "42", "-fmc", "2", "-gamma", "0.3", "-label", "3"]


@pytest.mark.parametrize("variant", ["dense", "sparse"])
def test_pt_driver_matches_reference_files(tmp_path, variant):
    sparse = variant == "sparse"
    flags = list(PT_FLAGS)
    if sparse:
        flags = [f if f != "12" else "16" for f in flags]
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    run([os.path.join(BIN, "pspin_pt_sparse" if sparse else "pspin_pt"), *flags], ours)
    run([os.path.join(REF, "parallel_tempering_sparse" if sparse else "parallel_tempering"), *flags], ref)
    d_o, d_r = the_dir(ours), the_dir(ref)
    assert os.path.basename(d_o) == os.path.basename(d_r)         # make_run_dir naming
    files_r = sorted(os.listdir(d_r))
    assert sorted(os.listdir(d_o)) == files_r
    same = ["params.txt", "temperatures.txt", "frequencies.txt"] + (["quartets.txt"] if sparse else [])
    for f in same:
        assert open(os.path.join(d_o, f)).read() == open(os.path.join(d_r, f)).read(), f
    assert open(os.path.join(d_o, "time.txt")).readline() == open(os.path.join(d_r, "time.txt")).readline()
    for f in ["energy_accept.txt", "exchanges.txt", "energy_split.txt"]:
        h_o, r_o = table(os.path.join(d_o, f))
        h_r, r_r = table(os.path.join(d_r, f))
        assert h_o == h_r, f
        assert len(r_o) == len(r_r), f
        assert [len(x) for x in r_o] == [len(x) for x in r_r], f
        assert [x[:3] for x in r_o] == [x[:3] for x in r_r], f      # sweep, Tidx, T columns
    assert os.path.getsize(os.path.join(d_o, "configs.bin")) == os.path.getsize(os.path.join(d_r, "configs.bin"))
    # exchange counts per window: same number of proposals
    _, ex_o = table(os.path.join(d_o, "exchanges.txt"))
    _, ex_r = table(os.path.join(d_r, "exchanges.txt"))
    assert [x[5] for x in ex_o] == [x[5] for x in ex_r]


def test_analysis_pt_reads_engine_output(tmp_path):
    flags = ["-N", "12", "-Tmax", "1.6", "-Tmin", "0.3", "-NT", "4", "-log_temp", "-nrep", "2", "-iter", "256",
             "-pt_freq", "1", "-save_freq", "16", "-seed", "7", "-label", "0", "-batch", "3"]
    run([os.path.join(BIN, "pspin_pt"), *flags], tmp_path)
    assert len(os.listdir(tmp_path / "data")) == 3                    # -batch 3: three sample dirs
    p = run([os.path.join(REF, "analysis_pt"), "-N", "12", "-NT", "4", "-nrep", "2", "--log-temp"], tmp_path)
    assert "samples" in p.stdout
    out = tmp_path / "analysis"
    produced = [f for _, _, fs in os.walk(out) for f in fs]
    assert len(produced) > 0, p.stdout[-2000:]


def test_mc_driver_matches_reference_files(tmp_path):
    flags = ["-N", "12", "-nrep", "3", "-T", "0.8", "-iter", "40", "-save_freq", "10", "-seed", "5", "-label", "1"]
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    run([os.path.join(BIN, "pspin_mc"), *flags], ours)
    run([os.path.join(REF, "pspin24"), *flags], ref)
    d_o, d_r = the_dir(ours), the_dir(ref)
    assert os.path.basename(d_o) == os.path.basename(d_r)
    h_o, r_o = table(os.path.join(d_o, "energy_accept.txt"))
    h_r, r_r = table(os.path.join(d_r, "energy_accept.txt"))
    assert h_o == h_r and len(r_o) == len(r_r) and [x[0] for x in r_o] == [x[0] for x in r_r]
    assert sorted(os.listdir(os.path.join(d_o, "configs"))) == sorted(os.listdir(os.path.join(d_r, "configs")))
    assert open(os.path.join(d_o, "time_per_iter.txt")).readline() == \
        open(os.path.join(d_r, "time_per_iter.txt")).readline()
    # the first saved energies agree at the start of the run only statistically;
    # check they are finite and the acceptance is a rate
    vals = np.array([[float(v) for v in x[1:]] for x in r_o])
    assert np.all(np.isfinite(vals)) and np.all((vals[:, 1::2] >= 0) & (vals[:, 1::2] <= 1))


def test_gpu_overlap_distribution_matches_analysis_pt(tmp_path):
    """P(q), the IFO P(C) and the experimental-IFO P(C) from the saved
    configurations on the GPU (pspin_overlap_counts, pspin_ifo_counts +
    cuda_pspin_b200.analysis) equal the reference analysis_pt's
    parisi_overlap.dat, ifo_overlap.dat and exp_ifo_overlap.dat on the same
    runs (same headers, bins, densities and jackknife errors, same
    temperatures), and the moments, glass-observable and per-sample <x^2>
    files derived from them are the reference's byte for byte."""
    flags = ["-N", "12", "-Tmax", "1.6", "-Tmin", "0.3", "-NT", "4", "-log_temp", "-nrep", "3", "-iter", "512",
             "-pt_freq", "1", "-save_freq", "8", "-seed", "11", "-label", "0", "-batch", "6"]
    run([os.path.join(BIN, "pspin_pt"), *flags], tmp_path)
    run([os.path.join(REF, "analysis_pt"), "-N", "12", "-NT", "4", "-nrep", "3", "--log-temp"], tmp_path)
    p = subprocess.run([sys.executable, "-m", "cuda_pspin_b200.analysis", "-N", "12", "-NT", "4", "-nrep", "3",
                        "--out", str(tmp_path / "gpu")], cwd=tmp_path, capture_output=True, text=True, timeout=300,
                       env={**os.environ, "PYTHONPATH": ROOT})
    assert p.returncode == 0, p.stderr[-2000:]
    for name in ("parisi_overlap.dat", "ifo_overlap.dat", "exp_ifo_overlap.dat"):
        refs = [os.path.join(r, f) for r, _, fs in os.walk(tmp_path / "analysis") for f in fs if f == name]
        assert len(refs) == 1, name
        ours = open(tmp_path / "gpu" / name).read().splitlines()
        theirs = open(refs[0]).read().splitlines()
        assert len(ours) == len(theirs), name
        n_rows = filled = 0
        for a, b in zip(ours, theirs):
            if a.startswith("#") or not a.strip():
                assert a == b, name
                continue
            x, y = np.array(a.split(), float), np.array(b.split(), float)
            assert x[0] == y[0] and x[3] == y[3], name
            assert abs(x[1] - y[1]) <= 1e-12 * max(1.0, abs(y[1])), (name, a, b)
            assert abs(x[2] - y[2]) <= 1e-9 * max(1.0, abs(y[2])), (name, a, b)
            n_rows += 1
            filled += y[1] > 0
        assert n_rows == 4 * 100 and filled > 4, name
    refdir = [r for r, _, fs in os.walk(tmp_path / "analysis") if "parisi_overlap.dat" in fs][0]
    for tag in ("parisi", "ifo", "exp_ifo"):
        for suffix in ("moments.dat", "glass_observables.dat", "sample_x2.dat"):
            name = f"{tag}_{suffix}"
            assert open(tmp_path / "gpu" / name).read() == open(os.path.join(refdir, name)).read(), name


SA_FLAGS = ["-N", "12", "-nrep", "3", "-Tmax", "1.6", "-Tmin", "0.3", "-ntemp", "5", "-iter", "6", "-save_freq", "16",
            "-seed", "9", "-fmc", "2", "-gamma", "0.3", "-label", "2"]


def test_sa_driver_matches_reference_files(tmp_path):
    """pspin_sa against the reference's simulated_annealing: same directory,
    same frequencies.txt and time.txt header, the same energy_accept.txt
    header, rows, temperature and sweep columns, and the same configuration
    files (second half of the schedule, conf_r{r}_T{T}.bin)."""
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    run([os.path.join(BIN, "pspin_sa"), *SA_FLAGS], ours)
    run([os.path.join(REF, "simulated_annealing"), *SA_FLAGS], ref)
    d_o, d_r = the_dir(ours), the_dir(ref)
    assert os.path.basename(d_o) == os.path.basename(d_r) == "SA_N12_NR3_S2"
    assert sorted(os.listdir(d_o)) == sorted(os.listdir(d_r))
    assert open(os.path.join(d_o, "frequencies.txt")).read() == open(os.path.join(d_r, "frequencies.txt")).read()
    assert open(os.path.join(d_o, "time.txt")).readline() == open(os.path.join(d_r, "time.txt")).readline()
    t_o = open(os.path.join(d_o, "time.txt")).read().split("\n")[1].split()[:6]
    t_r = open(os.path.join(d_r, "time.txt")).read().split("\n")[1].split()[:6]
    assert t_o == t_r                                                # N nrep ntemp sweeps/T Tmax Tmin
    h_o, r_o = table(os.path.join(d_o, "energy_accept.txt"))
    h_r, r_r = table(os.path.join(d_r, "energy_accept.txt"))
    assert h_o == h_r
    assert [x[:2] for x in r_o] == [x[:2] for x in r_r]              # T (%.8f) and sweep columns
    assert [len(x) for x in r_o] == [len(x) for x in r_r]
    confs = sorted(os.listdir(os.path.join(d_r, "configs")))
    assert len(confs) == 3 * 3 and sorted(os.listdir(os.path.join(d_o, "configs"))) == confs
    for f in confs:
        a = np.fromfile(os.path.join(d_o, "configs", f), np.float64)
        b = np.fromfile(os.path.join(d_r, "configs", f), np.float64)
        assert a.size == b.size == 2 * 12
        # same initial amplitudes and radius-conserving moves: each replica
        # stays on the sphere it started on (the reference's initial radius)
        assert abs(np.sum(a * a) - np.sum(b * b)) < 1e-5 * np.sum(b * b)


def test_analysis_sa_reads_engine_output(tmp_path):
    flags = ["-N", "12", "-nrep", "2", "-Tmax", "1.6", "-Tmin", "0.3", "-ntemp", "4", "-iter", "6",
             "-save_freq", "16", "-seed", "3", "-label", "0", "-batch", "3"]
    run([os.path.join(BIN, "pspin_sa"), *flags], tmp_path)
    assert sorted(os.listdir(tmp_path / "data")) == ["SA_N12_NR2_S0", "SA_N12_NR2_S1", "SA_N12_NR2_S2"]
    p = run([os.path.join(REF, "analysis_sa"), "-N", "12", "-nrep", "2"], tmp_path)
    assert "samples" in p.stdout
    produced = [f for _, _, fs in os.walk(tmp_path / "analysis") for f in fs]
    assert len(produced) > 0, p.stdout[-2000:]


def test_sa_statistics_match_reference(tmp_path):
    """Annealing the same 32 disorder samples (seeds 100..131, identical
    couplings and initial amplitudes) with pspin_sa -batch 32 and with 32 runs
    of the reference's simulated_annealing: for every temperature of the
    schedule, the mean over samples of (engine - reference) of the
    second-half window averages of E/N and of the acceptance is compared
    with its standard error.  The per-replica chains have the same law on
    both sides (the engine shares one pair schedule among a sample's
    replicas), so the paired z-scores are standard normal: every |z| < 3.5
    and at least 80 % within 2 sigma."""
    S, nrep, ntemp, it, save = 32, 4, 6, 9, 64
    flags = ["-N", "12", "-nrep", str(nrep), "-Tmax", "1.6", "-Tmin", "0.3", "-ntemp", str(ntemp),
             "-iter", str(it), "-save_freq", str(save)]
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    run([os.path.join(BIN, "pspin_sa"), *flags, "-seed", "100", "-label", "0", "-batch", str(S)], ours)
    for k in range(S):
        run([os.path.join(REF, "simulated_annealing"), *flags, "-seed", str(100 + k), "-label", str(k)], ref)

    def observables(path):
        rows = np.loadtxt(os.path.join(path, "energy_accept.txt"))
        Ts = np.unique(rows[:, 0])[::-1]
        assert len(Ts) == ntemp
        out = np.zeros((2, ntemp))
        for t, T in enumerate(Ts):
            blk = rows[(rows[:, 0] == T) & (rows[:, 1] > (1 << it) // 2)]
            out[0, t] = blk[:, 2::2].mean()
            out[1, t] = blk[:, 3::2].mean()
        return out

    names = [f"SA_N12_NR{nrep}_S{k}" for k in range(S)]
    obs_o = np.array([observables(str(ours / "data" / n)) for n in names])
    obs_r = np.array([observables(str(ref / "data" / n)) for n in names])
    diff = obs_o - obs_r
    z = diff.mean(axis=0) / (diff.std(axis=0, ddof=1) / np.sqrt(S))
    print("paired z (E/N, acc) per T:", np.round(z, 2).tolist())
    print("engine E/N per T:", np.round(obs_o[:, 0].mean(axis=0), 4).tolist())
    print("reference E/N per T:", np.round(obs_r[:, 0].mean(axis=0), 4).tolist())
    assert np.all(np.abs(z) < 3.5), z
    assert np.mean(np.abs(z) < 2.0) >= 0.8, z


@pytest.mark.parametrize("variant", ["dense", "sparse"])
def test_gpu_deeper_analysis_matches_analysis_pt(tmp_path, variant):
    """The deeper block on the GPU (pspin_deeper_counts, pspin_multi_overlap,
    the host sampling helpers and cuda_pspin_b200.analysis --deeper) against
    analysis_pt --deeper on the same runs: marginal_a2.dat, ipr.dat,
    ipr_sample.dat, the phase overlap with its moments, glass observables and
    per-sample <x^2>, for the sparse runs (quartets.txt) the link overlap
    files and the downsampled q-q_link scatter, the multi-overlap scatter
    file of every temperature, and decorrelation_time.dat -- byte for byte."""
    sparse = variant == "sparse"
    N = "16" if sparse else "12"
    flags = ["-N", N, "-Tmax", "1.6", "-Tmin", "0.3", "-NT", "4", "-log_temp", "-nrep", "3", "-iter", "1024",
             "-pt_freq", "1", "-save_freq", "8", "-seed", "21", "-label", "0", "-batch", "4"]
    if sparse:
        flags += ["-fmc", "1", "-gamma", "1"]
    run([os.path.join(BIN, "pspin_pt_sparse" if sparse else "pspin_pt"), *flags], tmp_path)
    run([os.path.join(REF, "analysis_pt"), "-N", N, "-NT", "4", "-nrep", "3", "--log-temp", "--deeper",
         *(["--sparse"] if sparse else [])], tmp_path)
    p = subprocess.run([sys.executable, "-m", "cuda_pspin_b200.analysis", "-N", N, "-NT", "4", "-nrep", "3",
                        "--deeper", "--out", str(tmp_path / "gpu")], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600, env={**os.environ, "PYTHONPATH": ROOT})
    assert p.returncode == 0, p.stderr[-2000:]
    refdir = [r for r, _, fs in os.walk(tmp_path / "analysis") if "phase_overlap.dat" in fs]
    assert len(refdir) == 1
    names = ["marginal_a2.dat", "ipr.dat", "ipr_sample.dat", "decorrelation_time.dat"]
    tags = ["phase", "link"] if sparse else ["phase"]
    for tag in tags:
        names += [f"{tag}_overlap.dat", f"{tag}_moments.dat", f"{tag}_glass_observables.dat",
                  f"{tag}_sample_x2.dat"]
    if sparse:
        names.append("scatter_q_qlink.dat")
    else:
        assert not os.path.exists(tmp_path / "gpu" / "link_overlap.dat")
    multi = sorted(f for f in os.listdir(refdir[0]) if f.startswith("multi_overlap_T"))
    assert len(multi) == 4
    names += multi
    differ = [n for n in names if open(tmp_path / "gpu" / n).read() != open(os.path.join(refdir[0], n)).read()]
    assert not differ, differ


@pytest.mark.parametrize("prog,extra", [("pspin_pt", ["-Tmax", "1.6", "-Tmin", "0.3", "-NT", "4", "-log_temp",
                                                     "-pt_freq", "1"]),
                                        ("pspin_sa", ["-Tmax", "1.6", "-Tmin", "0.3", "-ntemp", "4"])])
def test_sharded_driver_equals_unsharded(tmp_path, prog, extra):
    """-batch 5 split over three processes with -shard r/3 (each would run
    on its own GPU with -dev) writes the same five data directories as one
    unsharded -batch 5 run, file for file (time.txt aside)."""
    flags = ["-N", "12", "-nrep", "3", "-iter", "8" if prog == "pspin_sa" else "256", "-save_freq", "16",
             "-seed", "5", "-label", "0", "-batch", "5", *extra]
    one, split = tmp_path / "one", tmp_path / "split"
    one.mkdir()
    split.mkdir()
    run([os.path.join(BIN, prog), *flags], one)
    for r in range(3):
        run([os.path.join(BIN, prog), *flags, "-shard", f"{r}/3"], split)
    d1, d2 = sorted(os.listdir(one / "data")), sorted(os.listdir(split / "data"))
    assert d1 == d2 and len(d1) == 5
    for d in d1:
        for root, _, fs in os.walk(one / "data" / d):
            for f in fs:
                if f == "time.txt":
                    continue
                rel = os.path.relpath(os.path.join(root, f), one / "data" / d)
                a = open(os.path.join(root, f), "rb").read()
                b = open(split / "data" / d / rel, "rb").read()
                assert a == b, (d, rel)
