"""The reference's own programs, compiled unchanged against the engine.

oracle/Makefile (target `compat`) compiles the reference's test programs
(test_spherical.cu, test_inf_temp.cu, test_replica_exchange.cu,
test_detailed_balance.cu) and its PT drivers (parallel_tempering.cu,
parallel_tempering_sparse.cu, with config.cu) from their sources, with
include/compat/ in front of the reference's include directory, so that
their `#include "mc.h"` / `"mc_sparse.h"` resolve to the shim over
libpspin.so; the binaries land in oracle/_ref/compat/.

  * test_inf_temp and test_replica_exchange exit 0 (their own criteria);
    test_spherical and test_detailed_balance are compared with the
    reference's own builds of them (oracle/_ref/), since their bars assume
    FP64 amplitudes and compare two different disorder samples;
  * the reference's PT driver, running on the engine through the shim (its
    host exchange loop, its files, its cudaMemset of the counters through
    the shim's device pointers), writes files byte-identical to the
    engine's own driver pspin_pt, which runs the same chain with the
    exchange on the device: the same disorder, moves and drand48 exchange
    stream give the same trajectory.
"""
import filecmp
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COMPAT = os.path.join(ROOT, "oracle", "_ref", "compat")
BIN = os.path.join(ROOT, "cuda_pspin_b200", "bin")


def _need(name):
    path = os.path.join(COMPAT, name)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (make -C oracle compat needs the reference sources)")
    return path


REF = os.path.join(ROOT, "oracle", "_ref")


def _run_prog(path, cwd):
    p = subprocess.run([path], cwd=cwd, capture_output=True, text=True, timeout=900)
    return p.returncode, p.stdout + p.stderr


@pytest.mark.parametrize("prog", ["test_inf_temp", "test_replica_exchange"])
def test_reference_test_program_passes_on_the_engine(tmp_path, prog):
    rc, out = _run_prog(_need(prog), tmp_path)
    print(out[-1500:])
    assert rc == 0, out[-3000:]
    assert "FAIL" not in out.replace("SOME TESTS FAILED", "")


def _floats_after(text, key):
    return [float(line.split(key)[1].split()[0]) for line in text.splitlines() if key in line]


def test_reference_spherical_test_on_the_engine(tmp_path):
    """test_spherical checks |sum |a|^2 - N| <= 1e-8 after init and during
    500 sweeps, a bar for FP64 amplitudes.  The engine keeps FP32 amplitudes
    (FP64 only for the running energy, the resync and the renormalisation,
    every 1024 sweeps by default), so the program reports errors at FP32
    rounding: checked here to stay below 1e-4 (6e-6 of N), while the
    reference's own build of the same program passes its bar."""
    rc_e, out_e = _run_prog(_need("test_spherical"), tmp_path)
    ref = os.path.join(REF, "test_spherical")
    if os.path.exists(ref):
        rc_r, out_r = _run_prog(ref, tmp_path)
        assert rc_r == 0, out_r[-2000:]
    errs = _floats_after(out_e, "max |sum|a|^2 - N| =")
    print(out_e[-800:])
    assert len(errs) == 2 and max(errs) < 1e-4, errs


def test_reference_detailed_balance_test_on_the_engine(tmp_path):
    """test_detailed_balance compares <E/N> of two groups built from two
    different disorder samples (seeds 11111 and 99999) at N=8; different
    couplings give different equilibrium energies, so the program's 5-sigma
    verdict is not a property of the sampler.  What is: each group's <E/N>
    on the engine (same couplings and initial amplitudes bit for bit) equals
    the reference build's within 4 combined standard errors, and both builds
    reach the same verdict."""
    ref = os.path.join(REF, "test_detailed_balance")
    if not os.path.exists(ref):
        pytest.skip("reference test program not built")
    _, out_e = _run_prog(_need("test_detailed_balance"), tmp_path)
    _, out_r = _run_prog(ref, tmp_path)
    print("engine:", out_e[-600:], "reference:", out_r[-600:])
    for group in ("Group A:", "Group B:"):
        le = [l for l in out_e.splitlines() if group in l][0].split("=")[1].split("+/-")
        lr = [l for l in out_r.splitlines() if group in l][0].split("=")[1].split("+/-")
        me, se = float(le[0]), float(le[1])
        mr, sr = float(lr[0]), float(lr[1])
        assert abs(me - mr) <= 4.0 * (se * se + sr * sr) ** 0.5, (group, me, se, mr, sr)
    assert ("ALL PASSED" in out_e) == ("ALL PASSED" in out_r)


FLAGS = ["-Tmax", "1.5", "-Tmin", "0.3", "-NT", "6", "-log_temp", "-nrep", "4", "-iter", "2048",
         "-pt_freq", "1", "-save_freq", "64", "-seed", "77", "-label", "5"]


@pytest.mark.parametrize("variant,N,extra", [("dense", 12, ["-fmc", "2", "-gamma", "0.2"]),
                                             ("dense", 16, []),
                                             ("sparse", 16, ["-fmc", "1", "-gamma", "1"])])
def test_reference_driver_on_the_engine_equals_pspin_pt(tmp_path, variant, N, extra):
    ref_prog = "parallel_tempering_sparse" if variant == "sparse" else "parallel_tempering"
    ours_prog = "pspin_pt_sparse" if variant == "sparse" else "pspin_pt"
    flags = ["-N", str(N), *FLAGS, *extra]
    a, b = tmp_path / "shim", tmp_path / "ours"
    a.mkdir()
    b.mkdir()
    for prog, cwd in ((_need(ref_prog), a), (os.path.join(BIN, ours_prog), b)):
        p = subprocess.run([prog, *flags], cwd=cwd, capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    da, db = sorted(os.listdir(a / "data")), sorted(os.listdir(b / "data"))
    assert da == db and len(da) == 1
    fa, fb = a / "data" / da[0], b / "data" / db[0]
    files = sorted(set(os.listdir(fa)) - {"time.txt"})
    assert files == sorted(set(os.listdir(fb)) - {"time.txt"})
    assert "configs.bin" in files and "energy_accept.txt" in files
    differ = [f for f in files if not filecmp.cmp(fa / f, fb / f, shallow=False)]
    assert not differ, f"files differ: {differ}"
