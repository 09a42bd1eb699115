"""The smoothed-cube check (the reference's smoothed_cube.cu) on the engine.

pspin_smoothed_cube writes the reference's data files:
  * init_scatter.dat / moduli.dat: configurations from the reference's single
    cuRAND Philox call, scaled onto sum |a|^4 = N -- compared with the CPU
    oracle's restatement (cuRAND's host generator, which agrees with the
    device generator to an ulp, and the reference's scaling in FP64);
  * squircle.dat / superellipse.dat: the analytic boundaries;
  * mc_trajectory.dat: a free walk (no Hamiltonian) with the engine's FP32
    cube move: every saved point on sum |a|^4 = N to FP32 rounding, and the
    move's law -- t = |a_i|^4 / (|a_i|^4 + |a_j|^4) uniform after a move
    (spins_sparse.h:26-56) -- seen in the trajectory (N=2: t = |a_1|^4 / S4
    at every saved sweep, Kolmogorov-Smirnov against U(0,1)).
"""
import math
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROG = os.path.join(ROOT, "cuda_pspin_b200", "bin", "pspin_smoothed_cube")


def _load(path):
    return np.loadtxt(path, comments="#")


def _ks_uniform(x):
    x = np.sort(np.asarray(x))
    n = len(x)
    i = np.arange(1, n + 1)
    return max(np.max(i / n - x), np.max(x - (i - 1) / n))


@pytest.mark.parametrize("N", [2, 4])
def test_smoothed_cube_files(tmp_path, orc, N):
    nsamples, iter_, seed = 3000, 12, 42
    p = subprocess.run([PROG, "-N", str(N), "-iter", str(iter_), "-seed", str(seed), "-nsamples", str(nsamples)],
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    d = tmp_path / "smoothed_cube"
    # the reference's samples: normals (seed) scaled by (N / sum |a|^4)^(1/4)
    z = orc.curand_normals(seed, 2 * N * nsamples).reshape(nsamples, N, 2)
    r4 = np.sum((z[..., 0] ** 2 + z[..., 1] ** 2) ** 2, axis=1)
    a = z * ((N / r4) ** 0.25)[:, None, None]
    init = _load(d / "init_scatter.dat")
    mod = _load(d / "moduli.dat")
    np.testing.assert_allclose(init, a[:, :2, 0], rtol=0, atol=2e-8)
    np.testing.assert_allclose(mod, np.sqrt(a[:, :2, 0] ** 2 + a[:, :2, 1] ** 2), rtol=0, atol=2e-8)
    # boundaries
    s = N ** 0.25
    sq = _load(d / "squircle.dat")
    t = 2.0 * math.pi * np.arange(1001) / 1000
    np.testing.assert_allclose(sq[:, 0], np.where(np.cos(t) >= 0, 1.0, -1.0) * s * np.sqrt(np.abs(np.cos(t))),
                               atol=1e-8)
    se = _load(d / "superellipse.dat")
    t = 0.5 * math.pi * np.arange(501) / 500
    np.testing.assert_allclose(se[:, 1], s * np.sqrt(np.sin(t)), atol=1e-8)
    # free walk: 2^12 sweeps saved every 4 -> 1025 points on the constraint
    tr = _load(d / "mc_trajectory.dat")
    assert tr.shape == (1025, 6)
    assert tr[0, 0] == 0 and tr[-1, 0] == 4096
    assert np.all(np.abs(tr[:, 5] - N) < 1e-4 * N)
    if N == 2:
        tt = tr[1:, 3] ** 4 / tr[1:, 5]
        D = _ks_uniform(tt)
        print(f"N=2 walk: KS distance of |a1|^4/S4 from U(0,1) over {len(tt)} points: {D:.4f}")
        assert D < 1.95 / math.sqrt(len(tt))          # 0.1 % level
    else:
        assert np.std(tr[:, 1]) > 0.1 and np.std(tr[:, 2]) > 0.1
