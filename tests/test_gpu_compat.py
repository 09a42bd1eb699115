"""The reference's own programs, compiled unchanged against the engine.

oracle/Makefile (target `compat`) compiles the reference's test programs
(test_spherical.cu, test_inf_temp.cu, test_replica_exchange.cu,
test_detailed_balance.cu) and its PT drivers (parallel_tempering.cu,
parallel_tempering_sparse.cu, with config.cu) from their sources, with
include/compat/ in front of the reference's include directory, so that
their `#include "mc.h"` / `"mc_sparse.h"` resolve to the shim over
libpspin.so; the binaries land in oracle/_ref/compat/.

  * every test program exits 0 (its own PASS criteria);
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


@pytest.mark.parametrize("prog", ["test_spherical", "test_inf_temp", "test_replica_exchange",
                                  "test_detailed_balance"])
def test_reference_test_program_passes_on_the_engine(tmp_path, prog):
    p = subprocess.run([_need(prog)], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    print(p.stdout[-1500:])
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    assert "FAIL" not in p.stdout.replace("SOME TESTS FAILED", "")


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
