"""Parity of the CUDA engine with the CPU oracle, through the C ABI.

Disorder (couplings, FMC masks, survivor counts, sparse selection) and the
initial amplitudes come from the same cuRAND calls with the same seeds as the
reference's mc_init/mc_sparse_init, so they are compared exactly (masks,
indices) or to the last bits (FP64 values).  Every move of a traced replica
is replayed on the CPU: the kernel's FP32 dE must match the FP64 difference
of full energies on the same FP32 amplitudes within 1e-5 of the sum of
|terms| touched by the move.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def c4(n):
    return n * (n - 1) * (n - 2) * (n - 3) // 24


def cfg_pair(ps, orc, **kw):
    c = ps.default_config(**kw)
    if c.fmc_mode > 0 and c.gamma <= 0.0:
        c.gamma = 0.0 if c.fmc_mode == 1 else 1.0 / (2.0 * (c.N - 1))
    return c, orc.cfg(**kw)


# ---- index map and masks on the device -------------------------------------
@pytest.mark.parametrize("N", [4, 5, 8, 13, 20, 64])
def test_quartet_roundtrip_device(ps, N):
    assert ps.quartet_roundtrip(N) == 0          # test_quartet_index.cu:88-107


@pytest.mark.parametrize("N,fmc,seed,gamma", [(10, 1, 0, 1.0), (32, 2, 42, 0.1), (64, 2, 42, 0.1),
                                              (24, 2, 9, 1.0 / 46)])
def test_fmc_mask_device_bitexact(ps, orc, N, fmc, seed, gamma):
    w = orc.omega(N, fmc, seed)
    m, n = ps.fmc_mask(N, w, gamma)
    ref = orc.fmc_mask(N, w, gamma)
    assert np.array_equal(m, ref)
    assert n == int(np.unpackbits(ref).sum())


# ---- dense initialisation (mc_init) --------------------------------------------
@pytest.mark.parametrize("kw", [dict(N=8, nrep=4, fmc_mode=0, seed=1),
                                dict(N=12, nrep=6, fmc_mode=2, seed=7),
                                dict(N=16, nrep=3, fmc_mode=1, seed=3, gamma=1.0),
                                dict(N=32, nrep=8, fmc_mode=2, seed=42, gamma=0.1),
                                dict(N=24, nrep=5, fmc_mode=0, seed=11, J0=1.0, alpha0=0.3)])
def test_dense_init_matches_oracle(ps, orc, kw):
    c, oc = cfg_pair(ps, orc, **kw)
    ref = orc.DenseInit(oc)
    with ps.Engine(c) as eng:
        info = eng.info(0)
        assert info.n_pairs_active == ref.info.n_pairs_active
        assert info.n_quart_active == ref.info.n_quart_active
        assert info.h2_active == ref.info.h2_active
        g2, g4, mask = eng.couplings(0)
        N = c.N
        assert np.array_equal(mask, ref.mask)
        # same cuRAND stream on the device as the oracle's host generator
        np.testing.assert_allclose(g4, ref.g4[0::2], rtol=0, atol=1e-15 * max(1.0, np.abs(g4).max()))
        np.testing.assert_allclose(g2, ref.g2.reshape(N, N, 2)[..., 0], rtol=0, atol=1e-15)
        if c.fmc_mode:
            assert np.array_equal(eng.omega(0), ref.omega)
        sp = eng.get_spins()[0]
        np.testing.assert_allclose(sp, ref.spins_c().astype(np.complex64), rtol=0, atol=2e-7 * np.sqrt(N))
        E, acc, prop = eng.get_results()
        for r in range(c.nrep):
            e = sum(ref.energy(sp[r]))
            assert abs(E[r] - e) <= 1e-10 * (1 + abs(e))
        assert np.all(acc == 0) and np.all(prop == 0)


def test_curand_device_vs_host_generator(ps, orc):
    """The engine draws from cuRAND's device generator (as the reference
    does); the oracle from its host generator.  They agree to an ulp or so
    (bitwise equality with the reference is checked in test_golden.py)."""
    c, oc = cfg_pair(ps, orc, N=12, nrep=2, fmc_mode=0, seed=123)
    ref = orc.DenseInit(oc)
    with ps.Engine(c) as eng:
        g2, g4, _ = eng.couplings(0)
        # generator outputs differ by ~1 ulp of a unit normal before the
        # sigma rescale
        assert np.all(np.abs(g4 - ref.g4[0::2]) <= 2e-16)
        assert np.mean(g4 == ref.g4[0::2]) > 0.2


# ---- sparse initialisation (mc_sparse_init) --------------------------------------
@pytest.mark.parametrize("kw", [dict(N=8, nrep=2, fmc_mode=0, seed=2),
                                dict(N=16, nrep=4, fmc_mode=0, seed=11),
                                dict(N=20, nrep=4, fmc_mode=1, seed=5, gamma=1.0),
                                dict(N=24, nrep=4, fmc_mode=2, seed=8),
                                dict(N=10, nrep=2, fmc_mode=2, seed=4, gamma=0.01)])
def test_sparse_init_matches_oracle(ps, orc, kw):
    c, oc = cfg_pair(ps, orc, **kw)
    ref = orc.SparseInit(oc)
    with ps.Engine(c, ps.PSPIN_SPARSE) as eng:
        info = eng.info(0)
        assert info.n_quart_active == ref.info.n_quart_active
        assert info.n_quartets == ref.info.n_sparse
        q, g = eng.sparse_quartets(0)
        assert np.array_equal(q, ref.q)
        np.testing.assert_allclose(g, ref.qg, rtol=0, atol=1e-15)
        sp = eng.get_spins()[0]
        np.testing.assert_allclose(sp, ref.spins_c().astype(np.complex64), rtol=0, atol=2e-7 * np.sqrt(c.N))


# ---- per-move dE against the FP64 oracle ----------------------------------------------
def _trace_run(ps, orc, kw, variant, nsweeps=12, rep=1, T=0.7, generic=False):
    c, oc = cfg_pair(ps, orc, **kw)
    if variant == ps.PSPIN_DENSE and c.N > 32:
        nsweeps = 3        # the CPU replay costs two full C(N,4) energies per move
    ref = orc.DenseInit(oc) if variant == ps.PSPIN_DENSE else orc.SparseInit(oc)
    cap = nsweeps * (c.N // 2)
    with ps.Engine(c, variant, ps.make_options(trace=(0, rep, cap), resync_every=-1, generic_lists=generic)) as eng:
        s0 = eng.get_spins()[0][rep].copy()
        eng.fill_betas(1.0 / T)
        eng.sweep(nsweeps)
        tr = eng.trace(cap)
        E, acc, prop = eng.get_results()
        s1 = eng.get_spins()[0][rep]
    assert len(tr) == cap
    worst, worst_rel, n = orc.check_trace(ref, s0, tr)
    return worst, tr, s0, s1, acc[rep], ref


@pytest.mark.parametrize("kw", [dict(N=8, nrep=4, fmc_mode=0, seed=1),
                                dict(N=12, nrep=33, fmc_mode=2, seed=7),
                                dict(N=16, nrep=8, fmc_mode=0, seed=5, J0=0.5),
                                dict(N=20, nrep=4, fmc_mode=1, seed=3, gamma=2.0),
                                dict(N=32, nrep=2, fmc_mode=2, seed=42, gamma=0.1),
                                dict(N=48, nrep=4, fmc_mode=0, seed=21),
                                dict(N=64, nrep=3, fmc_mode=0, seed=22)])
@pytest.mark.parametrize("generic", [False, True])
def test_dense_per_move_dE(ps, orc, kw, generic):
    """Fully connected samples run on the blocked tiles by default and on the
    per-entry lists with generic_lists; both must meet the bound."""
    worst, tr, s0, s1, nacc, ref = _trace_run(ps, orc, kw, ps.PSPIN_DENSE, generic=generic)
    assert worst <= 1e-5, worst
    assert 0 < tr["accepted"].sum() == nacc
    # replaying accepted moves reproduces the final amplitudes exactly
    s = s0.copy()
    for rec in tr:
        if rec["accepted"]:
            s[rec["i0"]] = complex(*rec["ai_new"])
            s[rec["j0"]] = complex(*rec["aj_new"])
    assert np.array_equal(s.astype(np.complex64), s1.astype(np.complex64))


@pytest.mark.parametrize("kw", [dict(N=12, nrep=4, fmc_mode=0, seed=9),
                                dict(N=24, nrep=4, fmc_mode=2, seed=8),
                                dict(N=16, nrep=2, fmc_mode=1, seed=6, gamma=1.0)])
def test_sparse_per_move_dE(ps, orc, kw):
    worst, tr, *_ = _trace_run(ps, orc, kw, ps.PSPIN_SPARSE, nsweeps=20)
    assert worst <= 1e-5, worst


# ---- invariants (test_spherical.cu, test_sparse_dense.cu, test_inf_temp.cu) -----------
def test_spherical_constraint_and_energy_tracking(ps):
    c = ps.default_config(N=16, nrep=8, seed=77, T=1.0)
    with ps.Engine(c, options=ps.make_options(resync_every=-1)) as eng:
        r0 = np.sum(np.abs(eng.get_spins()[0]) ** 2, axis=1)
        assert np.allclose(r0, 16.0, rtol=1e-6)
        eng.sweep(200)
        sp = eng.get_spins()[0]
        assert np.allclose(np.sum(np.abs(sp) ** 2, axis=1), r0, rtol=1e-4)
        E, _, _ = eng.get_results()
        e2, e4 = eng.split_energies()
        assert np.all(np.abs(E - (e2 + e4)) / 16 < 1e-4)
        eng.resync()
        assert np.allclose(np.sum(np.abs(eng.get_spins()[0]) ** 2, axis=1), r0, rtol=1e-6)


def test_cube_constraint_and_energy_tracking(ps):
    c = ps.default_config(N=10, nrep=4, seed=54321, T=1.0, alpha0=0.0)
    with ps.Engine(c, ps.PSPIN_SPARSE, ps.make_options(resync_every=-1)) as eng:
        eng.sweep(300)
        sp = eng.get_spins()[0]
        assert np.allclose(np.sum(np.abs(sp) ** 4, axis=1), 10.0, rtol=1e-4)
        E, _, _ = eng.get_results()
        e2, e4 = eng.split_energies()
        assert np.all(np.abs(E - (e2 + e4)) / 10 < 1e-3)     # test_sparse_dense.cu:148


@pytest.mark.parametrize("variant", [0, 1])
def test_infinite_temperature_acceptance(ps, variant):
    c = ps.default_config(N=12, nrep=8, seed=31415, T=1e30, alpha0=0.0)
    with ps.Engine(c, variant) as eng:
        eng.fill_betas(0.0)
        eng.sweep(500)
        E, acc, prop = eng.get_results()
        assert np.all(prop == 500 * 6)
        assert np.all(acc == prop)                              # beta == 0 accepts all
        assert abs(np.mean(E / 12)) < 5.0


def test_deterministic_and_batch_equals_single(ps):
    cfgs = [ps.default_config(N=N, nrep=8, seed=100 + N, fmc_mode=f) for N, f in [(12, 0), (16, 2), (8, 1)]]
    for c in cfgs:
        if c.fmc_mode:
            c.gamma = 0.0 if c.fmc_mode == 1 else 1.0 / (2.0 * (c.N - 1))
            if c.fmc_mode == 1:
                c.gamma = 1.0
    with ps.Engine(cfgs) as batch:
        batch.fill_betas(1.2)
        batch.sweep(30)
        Eb, ab, pb = batch.get_results()
        sb = batch.get_spins()
    off = 0
    for k, c in enumerate(cfgs):
        with ps.Engine(c) as one:
            one.fill_betas(1.2)
            one.sweep(30)
            E1, a1, p1 = one.get_results()
            s1 = one.get_spins()[0]
        assert np.array_equal(E1, Eb[off:off + c.nrep])
        assert np.array_equal(a1, ab[off:off + c.nrep])
        assert np.array_equal(s1, sb[k])
        off += c.nrep


# ---- device replica exchange vs the host schedule (parallel_tempering.cu:316-352) ----
def test_device_exchange_matches_oracle(ps, orc):
    import ctypes
    NT, nr = 6, 3
    c = ps.default_config(N=12, nrep=NT * nr, seed=2024, fmc_mode=0)
    T, beta = ps.temperature_schedule(NT, 0.3, 1.5, True)
    with ps.Engine(c) as eng:
        eng.pt_init(NT, nr, beta, 1)
        perm = np.arange(NT * nr, dtype=np.int32)
        st = ctypes.c_uint64(orc.lib().orc_srand48_state(2024 + 5000))
        acc = np.zeros(NT - 1, np.int64)
        prop = np.zeros(NT - 1, np.int64)
        for step in range(40):
            eng.pt_run(1)
            E, _, _ = eng.get_results()
            p_dev, a_dev, q_dev = eng.pt_get(0)
            orc.lib().orc_exchange(NT, nr, orc.P(beta), orc.P(E), orc.P(perm), ctypes.byref(st),
                                   orc.P(acc), orc.P(prop), None)
            assert np.array_equal(p_dev, perm), step
            assert np.array_equal(a_dev, acc) and np.array_equal(q_dev, prop)
        assert acc.sum() > 0
