"""Pins of the CPU oracle against the reference's own known-answer tests.

The reference stores no golden vectors; its tests re-compute known answers
(src/test_quartet_index.cu, src/test_enum.cpp, src/test_fmc_mask.cu,
src/test_mean_shift.cu) or check invariants.  The same checks run here on the
oracle, plus published known-answer vectors for Philox4x32-10 (Random123) and
glibc's drand48 for the exchange stream.
"""
import ctypes
import itertools
import math

import numpy as np
import pytest


def c4(n):
    return n * (n - 1) * (n - 2) * (n - 3) // 24


# --- test_quartet_index.cu:88-131 ------------------------------------------
@pytest.mark.parametrize("N", range(4, 21))
def test_quartet_index_roundtrip(orc, N):
    L = orc.lib()
    i, j, k, l = (ctypes.c_int() for _ in range(4))
    q_enum = 0
    for ll in range(3, N):
        for kk in range(2, ll):
            for jj in range(1, kk):
                for ii in range(jj):
                    q = L.orc_encode_quartet(ii, jj, kk, ll)
                    assert q == q_enum
                    L.orc_decode_quartet(q, ctypes.byref(i), ctypes.byref(j), ctypes.byref(k), ctypes.byref(l))
                    assert (i.value, j.value, k.value, l.value) == (ii, jj, kk, ll)
                    q_enum += 1
    assert q_enum == c4(N) == L.orc_n_quartets(N)


# --- test_enum.cpp:15-102: 3-type enumeration == brute force ---------------
@pytest.mark.parametrize("N", [4, 5, 6, 8, 11, 14])
def test_three_type_enumeration(orc, N):
    L = orc.lib()
    for i0 in range(N):
        for j0 in range(i0 + 1, N):
            n = L.orc_three_type(N, i0, j0, None)
            out = np.zeros(4 * n, np.int32)
            L.orc_three_type(N, i0, j0, orc.P(out))
            got = sorted(map(tuple, out.reshape(-1, 4).tolist()))
            brute = sorted(q for q in itertools.combinations(range(N), 4) if i0 in q or j0 in q)
            assert got == brute


# --- FMC survivor known answers -----------------------------------------------
@pytest.mark.parametrize("N,fmc,seed,gamma,expect", [
    (10, 1, 42, 1.0, (0, 118, 0)),         # test_fmc_mask default arguments `10 1.0 1`
    (32, 1, 42, 1.0, (0, 6630, 0)),
    (32, 2, 42, 0.1, (255, 11955, 0)),      # dense PT configuration N=32, seed 42, gamma 0.1
])
def test_fmc_survivor_counts(orc, N, fmc, seed, gamma, expect):
    w = orc.omega(N, fmc, seed)
    cnt = (ctypes.c_int64 * 3)()
    tot = orc.lib().orc_count_survivors(N, orc.P(w), gamma, cnt)
    assert tuple(cnt) == expect and tot == sum(expect)
    m = orc.fmc_mask(N, w, gamma)
    assert orc.lib().orc_count_active_g4(orc.P(m), len(m)) == sum(expect)


def test_fmc_survivors_n64(orc):
    w = orc.omega(64, 2, 42)
    assert orc.lib().orc_count_survivors(64, orc.P(w), 0.1, None) == 214407


def _channel_py(w, q, gamma):
    i, j, k, l = q
    if abs(w[i] + w[j] - w[k] - w[l]) <= gamma:
        return 1
    if abs(w[i] + w[l] - w[j] - w[k]) <= gamma:
        return 2
    if abs(w[i] + w[k] - w[j] - w[l]) <= gamma:
        return 4
    return 0


@pytest.mark.parametrize("N,gamma", [(10, 1.0), (13, 0.7)])
def test_fmc_mask_matches_formula(orc, N, gamma):
    # test_fmc_mask.cu:75-78: srand48(42), omega = drand48()*N (glibc)
    libc = ctypes.CDLL("libc.so.6")
    libc.drand48.restype = ctypes.c_double
    libc.srand48(42)
    w = np.array([libc.drand48() * N for _ in range(N)])
    m = orc.fmc_mask(N, w, gamma)
    expect = [_channel_py(w, q, gamma) for q in
              sorted(itertools.combinations(range(N), 4), key=lambda t: (t[3], t[2], t[1], t[0]))]
    assert m.tolist() == expect


def test_fmc_g2_filter_matches_formula(orc):
    # test_fmc_mask.cu:137-159 (comb omega, gamma = 1.0)
    N, gamma = 10, 1.0
    c = orc.cfg(N=N, nrep=1, fmc_mode=1, seed=3, gamma=gamma)
    # comb: g2 never generated; uniform omega checks the filter itself
    c2 = orc.cfg(N=16, nrep=1, fmc_mode=2, seed=3, gamma=0.05)
    ref = orc.DenseInit(c2)
    g2 = ref.g2.reshape(16, 16, 2)[..., 0]
    w = ref.omega
    for i in range(16):
        for j in range(i + 1, 16):
            assert (g2[i, j] == 0.0) == (abs(w[i] - w[j]) > 0.05)
            assert g2[i, j] == g2[j, i]
    npa = sum(1 for i in range(16) for j in range(i, 16) if g2[i, j] != 0.0)
    assert npa == ref.info.n_pairs_active
    refc = orc.DenseInit(c)
    assert refc.info.n_pairs_active == 0 and refc.info.h2_active == 0


# --- Philox4x32-10 (Random123 known-answer vectors) ----------------------------
@pytest.mark.parametrize("ctr,key,out", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_kat(orc, ctr, key, out):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    orc.lib().orc_philox4x32_10(c, k, o)
    assert tuple(o) == out


# --- drand48: the exchange stream (parallel_tempering.cu:304, :334) ----------
@pytest.mark.parametrize("seed", [5042, 5000 + 2**33 + 7, 0])
def test_drand48_matches_glibc(orc, seed):
    libc = ctypes.CDLL("libc.so.6")
    libc.drand48.restype = ctypes.c_double
    libc.srand48(ctypes.c_long(seed))
    st = ctypes.c_uint64(orc.lib().orc_srand48_state(seed))
    for _ in range(1000):
        assert orc.lib().orc_drand48(ctypes.byref(st)) == libc.drand48()


# --- frequencies, schedule, seeds -------------------------------------------------
def test_omega_modes(orc):
    w = orc.omega(32, 2, 42)
    assert np.all(np.diff(w) >= 0) and w[0] >= 0 and w[-1] < 1
    st = ctypes.c_uint64(42 + 3000)
    raw = sorted((orc.lib().orc_splitmix64(ctypes.byref(st)) >> 11) / 2.0**53 for _ in range(32))
    assert np.array_equal(w, np.array(raw))
    assert np.array_equal(orc.omega(8, 1, 1), np.arange(8.0))


def test_auto_gamma(orc):
    L = orc.lib()
    assert L.orc_auto_gamma(1, 32, 0.0) == 0.0
    assert L.orc_auto_gamma(2, 32, 0.0) == 1.0 / 62.0
    assert L.orc_auto_gamma(2, 32, 0.1) == 0.1
    assert L.orc_auto_gamma(0, 32, 0.0) == 0.0


def test_temperature_schedule(orc):
    NT = 20
    T = np.zeros(NT)
    b = np.zeros(NT)
    orc.lib().orc_temperature_schedule(NT, 0.2, 1.6, 1, orc.P(T), orc.P(b))
    A = math.pow(0.2 / 1.6, 1.0 / (NT - 1))
    assert T[0] == 1.6 and abs(T[-1] - 0.2) < 1e-12
    assert all(T[t] == 1.6 * math.pow(A, t) for t in range(NT))
    orc.lib().orc_temperature_schedule(NT, 0.2, 1.6, 0, orc.P(T), orc.P(b))
    assert np.allclose(np.diff(T), -(1.4 / 19))


def test_replica_seeds(orc):
    out = np.zeros(4, np.uint64)
    orc.lib().orc_replica_seeds(42, 4, orc.P(out))
    st = ctypes.c_uint64(42)
    for r in range(4):
        assert int(out[r]) == orc.lib().orc_splitmix64(ctypes.byref(st))


# --- partial Fisher-Yates and sparse selection (mc_sparse.cu:340-349, 489-537)
def _splitmix(state):
    state = (state + 0x9e3779b97f4a7c15) & (2**64 - 1)
    z = state
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & (2**64 - 1)
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & (2**64 - 1)
    return state, z ^ (z >> 31)


def test_partial_shuffle(orc):
    arr = np.arange(1000, dtype=np.int64)
    orc.lib().orc_partial_shuffle(orc.P(arr), 1000, 37, 4042)
    ref = list(range(1000))
    st = 4042
    for i in range(37):
        st, r = _splitmix(st)
        j = i + r % (1000 - i)
        ref[i], ref[j] = ref[j], ref[i]
    assert arr.tolist() == ref


@pytest.mark.parametrize("N,fmc,gamma", [(9, 0, 0.0), (12, 1, 1.0), (14, 2, 0.08)])
def test_sparse_select_matches_enumeration(orc, N, fmc, gamma):
    seed = 99
    w = orc.omega(N, fmc, seed) if fmc else np.zeros(N)
    survivors = []
    for q, quad in enumerate(sorted(itertools.combinations(range(N), 4), key=lambda t: (t[3], t[2], t[1], t[0]))):
        m = 1 if fmc == 0 else _channel_py(w, quad, gamma)
        for ch in range(3):
            if m & (1 << ch):
                survivors.append(q * 3 + ch)
    ns = min(N, len(survivors))
    st = seed + 4000
    arr = list(survivors)
    for i in range(ns):
        st, r = _splitmix(st)
        j = i + r % (len(arr) - i)
        arr[i], arr[j] = arr[j], arr[i]
    out = np.zeros(N, np.int64)
    nnz = ctypes.c_int64()
    orc.lib().orc_sparse_select(N, orc.P(w), gamma, fmc, seed, N, orc.P(out), ctypes.byref(nnz))
    assert nnz.value == len(survivors)
    assert out[:ns].tolist() == arr[:ns]


# --- spin normalisation (spins.cu:27-69, spins_sparse.cu:28-61) ---------------
def _tree(vals, bd):
    s = list(vals) + [0.0] * (bd - len(vals))
    w = bd // 2
    while w > 0:
        for t in range(w):
            s[t] += s[t + w]
        w //= 2
    return s[0]


@pytest.mark.parametrize("N", [8, 12, 16, 24, 32, 48])
def test_sphere_normalisation_tree(orc, N):
    rng = np.random.default_rng(N)
    sp = rng.standard_normal(2 * N)
    a = sp.copy()
    orc.lib().orc_normalize_sphere(orc.P(a), N, 0)
    r2 = [sp[2 * i] ** 2 + sp[2 * i + 1] ** 2 for i in range(N)]
    scale = math.sqrt(N / _tree(r2, N))
    assert np.array_equal(a, sp * scale)
    radius = float(np.sum(a ** 2))
    if N & (N - 1) == 0:
        assert abs(radius - N) < 1e-10 * N
    b = sp.copy()
    orc.lib().orc_normalize_sphere(orc.P(b), N, 1)
    assert abs(np.sum(b ** 2) - N) < 1e-10 * N


@pytest.mark.parametrize("N", [16, 20, 40, 512])
def test_cube_normalisation(orc, N):
    rng = np.random.default_rng(N)
    sp = rng.standard_normal(2 * N)
    a = sp.copy()
    orc.lib().orc_normalize_cube(orc.P(a), N, 0)
    r4 = (a[0::2] ** 2 + a[1::2] ** 2) ** 2
    bd = max(32, (N + 31) // 32 * 32)
    if bd & (bd - 1) == 0:
        assert abs(r4.sum() - N) < 1e-9 * N


# --- test_mean_shift.cu: shift = J0_eff * N / n_surv on non-zero entries -----
def test_mean_shift(orc):
    N = 10
    base = orc.DenseInit(orc.cfg(N=N, nrep=1, fmc_mode=0, seed=5, J0=0.0))
    shifted = orc.DenseInit(orc.cfg(N=N, nrep=1, fmc_mode=0, seed=5, J0=1.5, alpha0=0.5))
    npa, nqa = base.info.n_pairs_active, base.info.n_quart_active
    m2 = 0.75 * N / npa
    m4 = 0.75 * N / nqa
    assert np.allclose(shifted.g2[0::2] - base.g2[0::2], m2, atol=1e-12)
    assert np.allclose(shifted.g4[0::2] - base.g4[0::2], m4, atol=1e-12)


def test_curand_host_deterministic(orc):
    a = orc.curand_normals(1234, 64)
    b = orc.curand_normals(1234, 64)
    assert np.array_equal(a, b) and abs(a.mean()) < 1.0
