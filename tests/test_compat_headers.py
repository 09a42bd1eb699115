"""CPU check that include/compat (the reference's mc.h / mc_sparse.h on top
of libpspin) compiles and links on its own: a program using every shim
call is compiled against a stand-in config.h that declares SimConfig with
the reference's field layout (config.h:9-25, the layout pspin_config
mirrors) and linked with libpspin.so.  Nothing is run (no GPU here); the
GPU test tests/test_gpu_compat.py runs the reference's own programs."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cuda_pspin_b200", "lib")

CONFIG_H = r"""
#pragma once
#include <cstdint>
struct SimConfig {
    int save_freq, verbose, N, nrep;
    double T, J, J0, alpha, alpha0;
    int mc_iterations;
    uint64_t seed;
    int label, dev, fmc_mode;
    double gamma;
};
"""

PROG = r"""
#include "mc_sparse.h"
#include <cstddef>
static_assert(sizeof(SimConfig) == sizeof(pspin_config), "SimConfig layout");
static_assert(offsetof(SparseQuartet, g) == 32, "SparseQuartet layout");
int main(int argc, char**) {
    if (argc > 5) {            // never taken: the calls only have to compile and link
        SimConfig c{};
        MCState d = mc_init(c);
        double e[4], b[4];
        long long a[4], p[4];
        cuDoubleComplex s[64];
        mc_set_betas(d, b);
        mc_sweep(d, c);
        mc_sweep_pt(d);
        mc_get_results(d, e, a, p);
        mc_get_spins(d, s);
        mc_compute_split_energies(d, e, b);
        mc_free(d);
        MCStateSparse q = mc_sparse_init(c);
        mc_sparse_set_betas(q, b);
        mc_sparse_sweep_pt(q);
        mc_sparse_get_results(q, e, a, p);
        mc_sparse_get_spins(q, s);
        mc_sparse_compute_split_energies(q, e, b);
        mc_sparse_free(q);
    }
    return 0;
}
"""


def test_compat_headers_compile_and_link(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc) or not os.path.exists(os.path.join(LIB, "libpspin.so")):
        pytest.skip("needs nvcc and a built libpspin.so")
    (tmp_path / "config.h").write_text(CONFIG_H)
    (tmp_path / "prog.cu").write_text(PROG)
    cmd = [nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include", "compat"), "-I", str(tmp_path), str(tmp_path / "prog.cu"),
           "-o", str(tmp_path / "prog"), "-L", LIB, "-lpspin"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
