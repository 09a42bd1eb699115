"""The drop-in drivers' argument errors against the reference's programs.

Both sides check their flags before any CUDA call, so this runs without a
GPU: for each bad command line the engine's driver and the reference's
program (rebuilt into oracle/_ref/) exit with the same code and print the
same first error line; the usage line is the reference's with the engine's
extension flags appended (parallel_tempering.cu:58-70,
simulated_annealing.cu:52-66, config.cu:45-58)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cuda_pspin_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")

CASES = [
    ("pspin_pt", "parallel_tempering", []),
    ("pspin_pt", "parallel_tempering", ["-N", "8", "-Tmax", "1", "-Tmin", "2", "-NT", "4", "-pt_freq", "1"]),
    ("pspin_pt", "parallel_tempering", ["-N", "8", "-Tmax", "2", "-Tmin", "1", "-NT", "1", "-pt_freq", "1"]),
    ("pspin_pt_sparse", "parallel_tempering_sparse", []),
    ("pspin_pt_sparse", "parallel_tempering_sparse", ["-N", "8", "-Tmax", "1", "-Tmin", "2", "-NT", "4",
                                                      "-pt_freq", "1"]),
    ("pspin_sa", "simulated_annealing", []),
    ("pspin_sa", "simulated_annealing", ["-N", "8", "-Tmax", "1", "-Tmin", "2", "-ntemp", "3"]),
    ("pspin_mc", "pspin24", ["-bogus", "3"]),
    ("pspin_smoothed_cube", "smoothed_cube", ["-bogus"]),
    ("pspin_smoothed_cube", "smoothed_cube", ["-N", "1"]),
    ("pspin_smoothed_cube", "smoothed_cube", ["-iter"]),
]


def _run(path, args, cwd):
    p = subprocess.run([path, *args], cwd=cwd, capture_output=True, text=True, timeout=60)
    return p.returncode, p.stderr.splitlines()


@pytest.mark.parametrize("ours,ref,args", CASES)
def test_argument_errors_match_reference(tmp_path, ours, ref, args):
    o, r = os.path.join(BIN, ours), os.path.join(REF, ref)
    if not (os.path.exists(o) and os.path.exists(r)):
        pytest.skip("drivers or reference programs not built")
    rc_o, err_o = _run(o, args, tmp_path)
    rc_r, err_r = _run(r, args, tmp_path)
    assert rc_o == rc_r != 0
    assert err_o and err_r and err_o[0].replace(o, "PROG") == err_r[0].replace(r, "PROG")
    if len(err_r) > 1:                       # usage: same text after the program name, extensions appended
        use_o = err_o[1].replace(o, "PROG")
        use_r = err_r[1].replace(r, "PROG")
        assert use_o.startswith(use_r), (use_o, use_r)
    assert not os.path.exists(tmp_path / "data") or not os.listdir(tmp_path / "data")


def test_sa_iteration_exponent_is_bounded(tmp_path):
    """-iter k gives 2^k sweeps per temperature; k above 30 is refused before
    any set-up (the reference shifts 1 << k unchecked)."""
    o = os.path.join(BIN, "pspin_sa")
    if not os.path.exists(o):
        pytest.skip("drivers not built")
    rc, err = _run(o, ["-N", "8", "-Tmax", "2", "-Tmin", "1", "-ntemp", "3", "-iter", "40"], tmp_path)
    assert rc == 1 and "-iter" in err[0]
