"""The C ABI library: loads without a GPU, exports every symbol that
include/pspin.h declares, and its host-only entry points (config defaults and
the reference's argv parser, config.h:28-46 and config.cu:6-70) behave like
the reference's.  No compute call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pspin.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pspin_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(ps):
    lib = ps.load_library()
    names = declared_symbols()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_config_matches_reference(ps):
    c = ps.default_config()
    assert (c.N, c.nrep, c.T, c.J, c.J0, c.alpha, c.alpha0) == (64, 1, 1.0, 2.0, 0.0, 0.5, 0.5)
    assert (c.mc_iterations, c.seed, c.save_freq, c.verbose, c.label, c.dev, c.fmc_mode, c.gamma) == \
        (10000, 42, 100, 0, -1, -1, 0, 0.0)
    assert ctypes.sizeof(ps.SimConfig) == 96      # SimConfig is 96 bytes


def test_parse_args(ps):
    c = ps.parse_args(["x", "-N", "32", "-nrep", "4", "-fmc", "2", "-seed", "17", "-verbose"])
    assert (c.N, c.nrep, c.fmc_mode, c.seed, c.verbose) == (32, 4, 2, 17, 1)
    assert c.gamma == 1.0 / 62.0                     # config.cu:61-67
    c = ps.parse_args(["x", "-fmc", "1", "-verbose", "2", "-gamma", "0.5"])
    assert (c.fmc_mode, c.gamma, c.verbose) == (1, 0.5, 2)
    c = ps.parse_args(["x", "-fmc", "1"])
    assert c.gamma == 0.0
    with pytest.raises(ps.PspinError) as e:
        ps.parse_args(["x", "-bogus"])
    assert "Unknown argument: -bogus" in str(e.value)
    with pytest.raises(ps.PspinError) as e:
        ps.parse_args(["x", "-N", "3"])
    assert "N must be >= 4" in str(e.value)


def test_version_and_error_string(ps):
    lib = ps.load_library()
    assert b"sm_100a" in lib.pspin_version()
    assert isinstance(lib.pspin_last_error(), bytes)


def test_bad_arguments_return_codes(ps):
    lib = ps.load_library()
    assert lib.pspin_create_batch(None, 0, 0, None, None) == 1
    assert lib.pspin_destroy(None) == 0


def test_host_exchange_matches_oracle(ps, orc):
    """pspin_exchange_host (the reference's host PT exchange, parallel_tempering.cu:316-352)
    equals the oracle's exchange, sample by sample, over many steps."""
    import ctypes
    rng = np.random.default_rng(3)
    S, NT, nr = 5, 6, 3
    beta = 1.0 / np.geomspace(1.5, 0.3, NT)
    rep_off = (np.arange(S, dtype=np.int64) * NT * nr)
    perm = np.tile(np.arange(NT * nr, dtype=np.int32), (S, 1))
    st = np.array([orc_srand(orc, 100 + k + 5000) for k in range(S)], np.uint64)
    acc = np.zeros((S, NT - 1), np.int64)
    prop = np.zeros((S, NT - 1), np.int64)
    betas = np.zeros(S * NT * nr)
    ref = [(perm[k].copy(), st[k:k + 1].copy(), np.zeros(NT - 1, np.int64), np.zeros(NT - 1, np.int64))
           for k in range(S)]
    for step in range(50):
        E = rng.normal(0, 3.0, S * NT * nr)
        ps.exchange_host(beta, E, rep_off, perm, st, acc, prop, betas)
        for k in range(S):
            p, s_, a_, pr_ = ref[k]
            bo = np.zeros(NT * nr)
            Ek = np.ascontiguousarray(E[k * NT * nr:(k + 1) * NT * nr])
            orc.lib().orc_exchange(NT, nr, orc.P(beta), orc.P(Ek), orc.P(p), orc.P(s_), orc.P(a_), orc.P(pr_),
                                   orc.P(bo))
            np.testing.assert_array_equal(perm[k], p)
            assert st[k] == s_[0]
            np.testing.assert_array_equal(acc[k], a_)
            np.testing.assert_array_equal(betas[k * NT * nr:(k + 1) * NT * nr], bo)
    assert acc.sum() > 0 and (prop == 50 * nr).all()


def orc_srand(orc, seed):
    return int(orc.lib().orc_srand48_state(seed))


def test_shard_samples_lpt(ps):
    """pspin_shard_samples: deterministic, complete, and within one largest
    cost of a perfect balance; equal samples go round robin."""
    rng = np.random.default_rng(3)
    Ns = rng.choice([24, 32, 48, 64], size=101)
    for n in (1, 2, 5, 8):
        of = ps.shard_samples(Ns, 96, n)
        assert np.array_equal(of, ps.shard_samples(Ns, 96, n))
        assert set(of.tolist()) <= set(range(n))
        loads = np.array([np.sum(Ns[of == r].astype(float) ** 4) for r in range(n)])
        assert loads.max() - loads.min() <= 64.0 ** 4
    assert ps.shard_samples([16] * 7, 4, 3).tolist() == [0, 1, 2, 0, 1, 2, 0]
    with pytest.raises(ps.PspinError):
        ps.shard_samples([16, 0], 4, 2)
