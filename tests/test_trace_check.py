"""CPU checks of the per-move replay that the GPU parity tests rely on
(oracle.check_trace): on a synthetic trace whose dE values are the FP64
energy differences rounded to FP32, it must report errors at FP32
rounding, a hamiltonian.cu-form difference equal to the g2 diagonal term,
and it must catch a planted error.  SparseFromList must give the sparse
set-up's energies for the same quartet list."""
import numpy as np
import pytest

REC = np.dtype([("i0", np.int32), ("j0", np.int32), ("ai_old", np.float32, 2), ("aj_old", np.float32, 2),
                ("ai_new", np.float32, 2), ("aj_new", np.float32, 2), ("dE", np.float32),
                ("accepted", np.int32), ("log_q_ratio", np.float32), ("log_u", np.float32)])


def _trace(ref, s0, n_moves, seed, plant=None):
    rng = np.random.default_rng(seed)
    s = s0.astype(np.complex64).astype(np.complex128)
    N = len(s)
    out = np.zeros(n_moves, REC)
    for m in range(n_moves):
        i0, j0 = sorted(rng.choice(N, 2, replace=False))
        new = s.copy()
        # the plain sphere move: keep |a_i|^2 + |a_j|^2, rotate phases
        r = abs(s[i0]) ** 2 + abs(s[j0]) ** 2
        t = rng.uniform(0.05, 0.95)
        new[i0] = np.sqrt(r * t) * np.exp(1j * rng.uniform(0, 2 * np.pi))
        new[j0] = np.sqrt(r * (1 - t)) * np.exp(1j * rng.uniform(0, 2 * np.pi))
        new = new.astype(np.complex64).astype(np.complex128)
        d = sum(ref.energy(new)) - sum(ref.energy(s))
        if plant is not None and m == plant:
            d *= 1.01
        acc = m % 3 != 0
        out[m] = (i0, j0, (s[i0].real, s[i0].imag), (s[j0].real, s[j0].imag), (new[i0].real, new[i0].imag),
                  (new[j0].real, new[j0].imag), d, int(acc), 0.0, 0.0)
        if acc:
            s = new
    return out


@pytest.mark.parametrize("N,fmc", [(10, 0), (10, 2), (64, 0)])
def test_check_trace_reports(orc, N, fmc):
    ref = orc.DenseInit(orc.cfg(N=N, nrep=1, fmc_mode=fmc, seed=5, gamma=0.3 if fmc else 0.0))
    s0 = ref.spins_c()[0].astype(np.complex64).astype(np.complex128)
    tr = _trace(ref, s0, 40, 1)
    rep = {}
    worst, rel, n = orc.check_trace(ref, s0, tr, report=rep)
    assert n == 40 and worst < 1e-6
    assert rep["rel_median"] <= rep["rel_max"] == rel
    assert rep["diag_max"] > 0.0          # the hamiltonian.cu form keeps g_ii |a_i|^2
    assert rep["ham_err_max"] < 1e-6      # dE32 + the diagonal term matches that form


def test_check_trace_catches_a_planted_error(orc):
    ref = orc.DenseInit(orc.cfg(N=10, nrep=1, fmc_mode=0, seed=6))
    s0 = ref.spins_c()[0].astype(np.complex64).astype(np.complex128)
    tr = _trace(ref, s0, 30, 2, plant=17)
    worst, _, _ = orc.check_trace(ref, s0, tr)
    assert worst > 1e-4


def test_sparse_from_list_matches_sparse_init(orc):
    ref = orc.SparseInit(orc.cfg(N=16, nrep=2, fmc_mode=1, seed=11, gamma=1.0))
    model = orc.SparseFromList(16, ref.q, ref.qg, ref.g2.reshape(16, 16, 2)[..., 0], ref.info.h2_active)
    for r in range(2):
        s = ref.spins_c()[r]
        assert model.energy(s) == ref.energy(s)
        new = s.copy()
        new[3] *= 1.1
        assert model.abs_terms(s, new, 3, 9) == ref.abs_terms(s, new, 3, 9)
