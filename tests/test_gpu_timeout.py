"""The sweep kernels' bounded waits, made to run out on purpose.

With the test option test_stall_move = k, every CTA of the ring-fed sweep
kernels waits at move k-1 of each launch on an mbarrier that nothing
completes, with the wait limit set by wait_limit_clocks.  The wait runs
out; the kernel must then stop issuing copies, drain the ones in flight,
return, and leave every replica as it was before the call: the call
returns PSPIN_ERR_TIMEOUT, amplitudes, energies and counters are
unchanged, the context stays usable, and the same handle built without the
stall runs normally.  No GPU fault, trap or endless wait is involved: each
wait gives up after about a millisecond.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STALL_CLOCKS = 2_000_000        # ~1 ms at 1.9 GHz


def _cfgs(ps):
    cfgs = [ps.default_config(N=N, nrep=40, seed=300 + k, fmc_mode=f) for k, (N, f) in
            enumerate(((12, 0), (16, 2), (20, 0)))]
    for c in cfgs:
        if c.fmc_mode == 2:
            c.gamma = 0.1
    return cfgs


def _state(eng):
    E, acc, prop = eng.get_results()
    return [s.copy() for s in eng.get_spins()], E.copy(), acc.copy(), prop.copy()


@pytest.mark.parametrize("cluster,warps,proposal", [(1, 4, 0), (2, 4, 0), (4, 2, 0), (1, 4, 1), (2, 2, 1)])
def test_stalled_wait_aborts_and_keeps_state(ps, cluster, warps, proposal):
    opts = ps.make_options(resync_every=-1, cluster_size=cluster, warps_per_unit=warps,
                           wait_limit_clocks=STALL_CLOCKS, test_stall_move=3)
    with ps.Engine(_cfgs(ps), ps.PSPIN_DENSE, opts) as eng:
        if proposal:
            eng.learn_init(seed=4, capacity=1024, record_prob=0.0)
            eng.set_proposal(proposal)
        eng.fill_betas(1.3)
        before = _state(eng)
        with pytest.raises(ps.PspinError) as ei:
            eng.sweep(2)
        assert ei.value.code == ps.PSPIN_ERR_TIMEOUT, str(ei.value)
        assert "kept their state" in str(ei.value)
        after = _state(eng)
        for x, y in zip(before[0], after[0]):
            np.testing.assert_array_equal(x, y)
        for i in (1, 2, 3):
            np.testing.assert_array_equal(before[i], after[i])
        # the context and the handle still work: FP64 energies of the kept state
        e2, e4 = eng.split_energies()
        np.testing.assert_allclose(after[1], e2 + e4, rtol=0, atol=1e-4 * np.abs(e2 + e4).max())

    # the same samples without the stall sweep normally on the same device
    opts = ps.make_options(resync_every=-1, cluster_size=cluster, warps_per_unit=warps)
    with ps.Engine(_cfgs(ps), ps.PSPIN_DENSE, opts) as eng:
        if proposal:
            eng.learn_init(seed=4, capacity=1024, record_prob=0.0)
            eng.set_proposal(proposal)
        eng.fill_betas(1.3)
        eng.sweep(2)
        E, acc, prop = eng.get_results()
        assert np.all(prop == 2 * np.repeat([6, 8, 10], 40))
        assert not np.array_equal(eng.get_spins()[0], before[0][0])


def test_stall_after_the_launch_changes_nothing(ps):
    """A stall move beyond the launch's last move is never reached: the
    launch completes and equals one without the option, bit for bit."""
    out = []
    for stall in (0, 10_000):
        opts = ps.make_options(resync_every=-1, cluster_size=2, warps_per_unit=4,
                               wait_limit_clocks=STALL_CLOCKS, test_stall_move=stall)
        with ps.Engine(_cfgs(ps), ps.PSPIN_DENSE, opts) as eng:
            eng.fill_betas(1.3)
            eng.sweep(3)
            out.append(_state(eng))
    for x, y in zip(out[0][0], out[1][0]):
        np.testing.assert_array_equal(x, y)
    for i in (1, 2, 3):
        np.testing.assert_array_equal(out[0][i], out[1][i])
