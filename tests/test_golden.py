"""Golden fixtures produced by the reference itself (tests/golden/make_golden.py
runs the reference's mc_init / mc_sparse_init, rebuilt for sm_100a, on a
B200).

CPU: the oracle reproduces them -- index-valued results (FMC masks, survivor
counts, frequencies, the sparse quartet selection) exactly, FP64 values to the
last bits (the oracle draws from cuRAND's host generator, the reference from
its device generator; the two differ by at most an ulp or so).
GPU: the engine reproduces them -- index-valued results exactly and the
couplings bit for bit (same device cuRAND stream).
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
NAMES = [os.path.basename(f)[:-4] for f in FILES]


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def kw_of(g):
    info = g["info"]
    N, R, fmc, gamma = int(info[0]), int(info[1]), int(info[2]), float(info[3])
    return N, R, fmc, gamma


SEEDS = {"s7": 7, "s3": 3, "s11": 11, "s5": 5, "s42": 42, "s9": 9, "s8": 8}
EXTRA = {"dense_n16_j0_s9": dict(J0=1.0, alpha0=0.3)}


def cfg_kw(name, g):
    N, R, fmc, gamma = kw_of(g)
    kw = dict(N=N, nrep=R, fmc_mode=fmc, gamma=gamma, seed=SEEDS[name.split("_")[-1]])
    kw.update(EXTRA.get(name, {}))
    return kw


def test_fixtures_present():
    assert len(FILES) >= 9


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_reference(orc, name):
    g = load(name)
    kw = cfg_kw(name, g)
    if kw["N"] > 64:
        pytest.skip("large sparse fixture: checked through orc_sparse_select in the GPU suite")
    dense = name.startswith("dense")
    ref = orc.DenseInit(orc.cfg(**kw)) if dense else orc.SparseInit(orc.cfg(**kw))
    info = g["info"]
    assert ref.info.n_pairs_active == int(info[4])
    assert ref.info.n_quart_active == int(info[5])
    assert ref.info.h2_active == int(info[6])
    N = kw["N"]
    if "omega" in g:
        assert np.array_equal(ref.omega, g["omega"])
    np.testing.assert_allclose(ref.g2.reshape(N, N, 2)[..., 0], g["g2"], rtol=0, atol=2e-15 * max(1, np.abs(g["g2"]).max()))
    if dense:
        assert np.array_equal(ref.mask, g["mask"])
        g4 = ref.g4[0::2][g["g4_active_q"]]
        np.testing.assert_allclose(g4, g["g4_active"], rtol=0, atol=2e-15 * max(1, np.abs(g4).max()))
    else:
        assert ref.info.n_sparse == int(info[7])
        assert np.array_equal(ref.q, g["quartets"])
        np.testing.assert_allclose(ref.qg, g["quartets_g"], rtol=0, atol=2e-15)
    np.testing.assert_allclose(ref.spins_c(), g["spins"], rtol=0, atol=4e-15 * np.sqrt(N))
    np.testing.assert_allclose(ref.energies, g["energies"], rtol=0, atol=1e-13 * N)


def test_oracle_sparse_selection_n512(orc):
    """mc_sparse_init's selection at N=512, comb, gamma=1: the oracle walks
    the 2.83e9 quartets in q order without storing them and must pick the
    reference's 512 (quartet, channel) pairs out of its 33,130,110 survivors."""
    import ctypes
    g = load("sparse_n512_fmc1_s42")
    N = 512
    w = orc.omega(N, 1, 42)
    enc = np.zeros(N, np.int64)
    nnz = ctypes.c_int64()
    assert orc.lib().orc_sparse_select(N, orc.P(w), 1.0, 1, 42, N, orc.P(enc), ctypes.byref(nnz)) == 0
    assert nnz.value == int(g["info"][5]) == 33130110
    L = orc.lib()
    i, j, k, l = (ctypes.c_int() for _ in range(4))
    got = []
    for e in enc:
        L.orc_decode_quartet(int(e) // 3, ctypes.byref(i), ctypes.byref(j), ctypes.byref(k), ctypes.byref(l))
        got.append((i.value, j.value, k.value, l.value, int(e) % 3))
    assert np.array_equal(np.array(got, np.int32), g["quartets"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_engine_reproduces_reference(ps, orc, name):
    g = load(name)
    kw = cfg_kw(name, g)
    dense = name.startswith("dense")
    c = ps.default_config(**kw)
    info = g["info"]
    with ps.Engine(c, ps.PSPIN_DENSE if dense else ps.PSPIN_SPARSE) as eng:
        i = eng.info(0)
        assert (i.n_pairs_active, i.n_quart_active, i.h2_active) == (int(info[4]), int(info[5]), int(info[6]))
        N = kw["N"]
        g2, g4, mask = eng.couplings(0, dense_g4=dense)
        assert np.array_equal(g2, g["g2"])                      # same device cuRAND stream: bitwise
        if "omega" in g:
            assert np.array_equal(eng.omega(0), g["omega"])
        if dense:
            assert np.array_equal(mask, g["mask"])
            assert np.array_equal(g4[g["g4_active_q"]], g["g4_active"])
        else:
            q, qg = eng.sparse_quartets(0)
            assert i.n_quartets == int(info[7])
            assert np.array_equal(q, g["quartets"])
            assert np.array_equal(qg, g["quartets_g"])
        sp = eng.get_spins()[0]
        ref32 = g["spins"].astype(np.complex64)
        # FP32 amplitudes: the reference's FP64 amplitudes rounded (ties of
        # a last-ulp normalisation difference allowed)
        np.testing.assert_allclose(sp, ref32, rtol=0, atol=2.5e-7 * np.sqrt(N))
        E, _, _ = eng.get_results()
        np.testing.assert_allclose(E, g["energies"], rtol=0, atol=1e-5 * N)
