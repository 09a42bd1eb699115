"""Generates the golden fixtures in this directory from the reference itself.

Runs oracle/_ref/ref_dump (the reference's mc_init / mc_sparse_init rebuilt
for sm_100a from its own sources by oracle/Makefile) on a GPU for the
configurations below and packs its state into compressed .npz files:

    python tests/golden/make_golden.py --out tests/golden

Each file holds: info (N, nrep, fmc, gamma, n_pairs_active, n_quart_active,
h2_active, n_quartets), the FMC mask (packed bits), g2 (real parts), g4 real
parts at the active quartets (dense), the sparse quartet list (sparse),
omega, the initial amplitudes and initial energies.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")

CONFIGS = [
    ("dense_n12_fmc2_s7", "dense", ["-N", "12", "-nrep", "6", "-fmc", "2", "-seed", "7"]),
    ("dense_n16_fmc0_s3", "dense", ["-N", "16", "-nrep", "4", "-fmc", "0", "-seed", "3"]),
    ("dense_n24_fmc0_s11", "dense", ["-N", "24", "-nrep", "4", "-fmc", "0", "-seed", "11"]),
    ("dense_n20_fmc1_s5", "dense", ["-N", "20", "-nrep", "3", "-fmc", "1", "-gamma", "1.0", "-seed", "5"]),
    ("dense_n32_fmc2_s42", "dense", ["-N", "32", "-nrep", "4", "-fmc", "2", "-gamma", "0.1", "-seed", "42"]),
    ("dense_n16_j0_s9", "dense", ["-N", "16", "-nrep", "2", "-fmc", "0", "-seed", "9", "-J0", "1.0",
                                  "-alpha0", "0.3"]),
    ("sparse_n16_fmc0_s11", "sparse", ["-N", "16", "-nrep", "4", "-fmc", "0", "-seed", "11"]),
    ("sparse_n24_fmc2_s8", "sparse", ["-N", "24", "-nrep", "4", "-fmc", "2", "-seed", "8"]),
    ("sparse_n20_fmc1_s5", "sparse", ["-N", "20", "-nrep", "2", "-fmc", "1", "-gamma", "1.0", "-seed", "5"]),
]
# the reference's N=512 sparse set-up needs ~48 GB of device and ~71 GB of
# host memory (a dense C(512,4) temporary); generated only with --big
BIG = [("sparse_n512_fmc1_s42", "sparse", ["-N", "512", "-nrep", "4", "-fmc", "1", "-gamma", "1.0",
                                           "-seed", "42"])]


def c4(n):
    return n * (n - 1) * (n - 2) * (n - 3) // 24


def pack(d: str, variant: str) -> dict:
    info = open(os.path.join(d, "info.txt")).read().split()
    N, R = int(info[0]), int(info[1])
    out = {"info": np.array([float(x) for x in info])}
    out["g2"] = np.fromfile(os.path.join(d, "g2.f64")).reshape(N, N, 2)[..., 0].copy()
    sp = np.fromfile(os.path.join(d, "spins.f64")).reshape(R, N, 2)
    out["spins"] = sp[..., 0] + 1j * sp[..., 1]
    out["energies"] = np.fromfile(os.path.join(d, "energies.f64"))
    if os.path.exists(os.path.join(d, "omega.f64")):
        out["omega"] = np.fromfile(os.path.join(d, "omega.f64"))
    if variant == "dense":
        mask = np.fromfile(os.path.join(d, "mask.u8"), np.uint8)
        g4 = np.fromfile(os.path.join(d, "g4.f64"))[0::2]
        assert len(mask) == c4(N)
        out["mask"] = mask
        active = np.nonzero(mask)[0]
        out["g4_active_q"] = active.astype(np.int64)
        out["g4_active"] = g4[active]
    else:
        q = np.loadtxt(os.path.join(d, "quartets.txt"), ndmin=2)
        out["quartets"] = q[:, :5].astype(np.int32)
        out["quartets_g"] = q[:, 5].copy()
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--big", action="store_true")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    todo = CONFIGS + (BIG if a.big else [])
    for name, variant, flags in todo:
        with tempfile.TemporaryDirectory() as tmp:
            subprocess.run([DUMP, tmp, variant, *flags], check=True, stdout=subprocess.DEVNULL)
            np.savez_compressed(os.path.join(a.out, name + ".npz"), **pack(tmp, variant))
        print("wrote", name)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
