"""Checkpoint / resume: a chain saved, reloaded into a fresh handle built
from the same configurations and continued equals the uninterrupted chain
bit for bit (amplitudes, energies, counters, PT permutation and exchange
counters), for the plain move and for the learned move."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NT, NR = 4, 2


def _engine(ps):
    cfgs = [ps.default_config(N=N, nrep=NT * NR, seed=90 + k, fmc_mode=2) for k, N in enumerate((12, 14))]
    for c in cfgs:
        c.gamma = 0.1
    eng = ps.Engine(cfgs, ps.PSPIN_DENSE, ps.make_options(resync_every=16))
    return eng


def _state(eng):
    E, acc, prop = eng.get_results()
    return eng.get_spins(), E, acc, prop, [eng.pt_get(k) for k in range(eng.n_samples)]


def _same(a, b):
    for x, y in zip(a[0], b[0]):
        np.testing.assert_array_equal(x, y)
    for i in (1, 2, 3):
        np.testing.assert_array_equal(a[i], b[i])
    for u, v in zip(a[4], b[4]):
        for x, y in zip(u, v):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("learned", [False, True])
def test_checkpoint_resume_is_bit_exact(ps, tmp_path, learned):
    path = str(tmp_path / "ck.bin")
    T, beta = ps.temperature_schedule(NT, 0.3, 1.5, True)
    with _engine(ps) as a:
        a.pt_init(NT, NR, beta, 1)
        if learned:
            a.learn_init(seed=3, capacity=4096, record_prob=0.5)
            a.set_proposal(ps.PROPOSAL_PLAIN_FIELDS)
            a.pt_run(20)
            a.learn_train(50, 512, 3e-3)
            a.set_proposal(ps.PROPOSAL_LEARNED)
        a.pt_run(27)                  # mid-way between resyncs (every 16 sweeps)
        a.checkpoint_save(path)
        a.pt_run(40)
        want = _state(a)
    with _engine(ps) as b:
        b.checkpoint_load(path)
        b.pt_run(40)
        got = _state(b)
    _same(want, got)


def test_checkpoint_rejects_other_handles(ps, tmp_path):
    path = str(tmp_path / "ck.bin")
    with _engine(ps) as a:
        a.checkpoint_save(path)
    c = ps.default_config(N=12, nrep=NT * NR, seed=91, fmc_mode=2)
    with ps.Engine(c) as b:
        with pytest.raises(ps.PspinError):
            b.checkpoint_load(path)
    with _engine(ps) as b:
        with pytest.raises(ps.PspinError):
            b.checkpoint_load(str(tmp_path / "missing.bin"))


def test_truncated_checkpoint_leaves_the_handle_unchanged(ps, tmp_path):
    """The whole file is read and checked before anything is written."""
    path = str(tmp_path / "ck.bin")
    T, beta = ps.temperature_schedule(NT, 0.3, 1.5, True)
    with _engine(ps) as a:
        a.pt_init(NT, NR, beta, 1)
        a.pt_run(9)
        a.checkpoint_save(path)
    raw = open(path, "rb").read()
    for cut in (len(raw) - 8, len(raw) // 2, 200):
        bad = str(tmp_path / f"cut{cut}.bin")
        open(bad, "wb").write(raw[:cut])
        with _engine(ps) as b:
            b.pt_init(NT, NR, beta, 1)
            b.pt_run(5)
            before = _state(b)
            with pytest.raises(ps.PspinError):
                b.checkpoint_load(bad)
            _same(before, _state(b))
    longer = str(tmp_path / "long.bin")
    open(longer, "wb").write(raw + b"\0")
    with _engine(ps) as b:
        with pytest.raises(ps.PspinError):
            b.checkpoint_load(longer)


def test_checkpoint_without_pt_drops_the_handles_pt_state(ps, tmp_path):
    """A chain saved before any PT set-up, loaded into a handle that has PT
    state, continues as the saved chain: plain sweeps equal, and the PT
    state is gone (pspin_pt_run needs a new pspin_pt_init)."""
    path = str(tmp_path / "ck.bin")
    T, beta = ps.temperature_schedule(NT, 0.3, 1.5, True)
    with _engine(ps) as a:
        a.fill_betas(1.1)
        a.sweep(7)
        a.checkpoint_save(path)
        a.sweep(11)
        E_a, acc_a, _ = a.get_results()
        s_a = a.get_spins()
    with _engine(ps) as b:
        b.pt_init(NT, NR, beta, 1)
        b.pt_run(3)
        b.checkpoint_load(path)
        with pytest.raises(ps.PspinError):
            b.pt_run(1)
        b.sweep(11)
        E_b, acc_b, _ = b.get_results()
        s_b = b.get_spins()
    np.testing.assert_array_equal(E_a, E_b)
    np.testing.assert_array_equal(acc_a, acc_b)
    for x, y in zip(s_a, s_b):
        np.testing.assert_array_equal(x, y)
