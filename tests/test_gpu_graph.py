"""The PT cycle replayed as a CUDA graph equals direct launches bit for bit,
and the block-shape autotuner leaves the chain where it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NT, NR = 4, 2


def _engine(ps, graph_steps, proposal=0, warps=0, cluster=None):
    # cluster None: default; 0: the list-resident kernel (as the autotuner reports it)
    cluster = 0 if cluster is None else (-1 if cluster == 0 else cluster)
    cfgs = [ps.default_config(N=N, nrep=NT * NR, seed=70 + k, fmc_mode=2) for k, N in enumerate((12, 16, 13))]
    for c in cfgs:
        c.gamma = 0.1
    eng = ps.Engine(cfgs, ps.PSPIN_DENSE, ps.make_options(resync_every=20, graph_steps=graph_steps,
                                                          warps_per_unit=warps, cluster_size=cluster))
    T, beta = ps.temperature_schedule(NT, 0.3, 1.5, True)
    eng.pt_init(NT, NR, beta, 1)
    if proposal:
        eng.learn_init(seed=4, capacity=4096, record_prob=0.25)
        eng.set_proposal(proposal)
    eng.observe_init(2, 200)
    return eng


def _state(ps, eng):
    E, acc, prop = eng.get_results()
    pts = [eng.pt_get(k) for k in range(eng.n_samples)]
    obs = eng.observe_get()
    return eng.get_spins(), E, acc, prop, pts, obs


@pytest.mark.parametrize("proposal", [0, 1])
def test_graph_replay_equals_direct_launches(ps, proposal):
    out = []
    for g in (8, -1):
        with _engine(ps, g, proposal) as eng:
            eng.pt_run(50)                 # crosses resyncs at 20 and 40, graphs of 8 steps between
            eng.pt_run(37)
            out.append(_state(ps, eng))
            if proposal:
                out[-1] = out[-1] + (eng.learn_records(4096),)
    a, b = out
    for x, y in zip(a[0], b[0]):
        np.testing.assert_array_equal(x, y)
    for i in (1, 2, 3):
        np.testing.assert_array_equal(a[i], b[i])
    for (p1, e1, f1), (p2, e2, f2) in zip(a[4], b[4]):
        np.testing.assert_array_equal(p1, p2)
        np.testing.assert_array_equal(e1, e2)
        np.testing.assert_array_equal(f1, f2)
    np.testing.assert_array_equal(a[5][0], b[5][0])
    np.testing.assert_array_equal(a[5][1], b[5][1])
    assert a[5][0].shape[0] == 87
    if proposal:
        assert a[6][0] == b[6][0] and a[6][0] > 0


def test_autotune_restores_the_chain(ps):
    with _engine(ps, -1) as eng:
        w, c, ms = eng.autotune(4)                 # first choice, on a fresh chain
    with _engine(ps, -1, warps=w, cluster=c) as eng:
        eng.pt_run(10)
        before = _state(ps, eng)
        w2, c2, ms = eng.autotune(4)
        after = _state(ps, eng)
        assert w2 in (1, 2, 4, 8) and c2 in (0, 1, 2, 4, 8, 16)
        ok = ms > 0
        assert ok[1].all() and ok[0, 0]            # every warp count without a cluster, and the resident kernel
        assert ms[[0, 1, 2, 4, 8, 16].index(c2), [1, 2, 4, 8].index(w2)] == ms[ok].min()
        for x, y in zip(before[0], after[0]):
            np.testing.assert_array_equal(x, y)
        for i in (1, 2, 3):
            np.testing.assert_array_equal(before[i], after[i])
        eng.pt_run(25)
        a = _state(ps, eng)
    if (w2, c2) != (w, c):
        return                                     # timings too close to give the same choice twice
    with _engine(ps, -1, warps=w, cluster=c) as eng:   # same block shape throughout, no autotune
        eng.pt_run(35)
        b = _state(ps, eng)
    for x, y in zip(a[0], b[0]):                   # so the sweep index was restored too
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a[1], b[1])


def test_tensor_core_resync(ps):
    """Periodic energies from the split-BF16 contraction: the running energy
    after a resync equals the FP64 energy to the contraction's accuracy, and
    the recorded drift is the FP32 accumulation error before it."""
    c = ps.default_config(N=24, nrep=32, seed=5, fmc_mode=0, T=0.5)
    with ps.Engine(c, ps.PSPIN_DENSE, ps.make_options(resync_every=16, resync_method=ps.RESYNC_TC)) as eng:
        eng.fill_betas(2.0)
        eng.sweep(64)                              # four resyncs, the last one at sweep 64
        E, _, _ = eng.get_results()
        e2, e4 = eng.split_energies()              # FP64 of the same amplitudes
        drift = eng.resync_drift()
    ref = e2 + e4
    scale = np.abs(ref).max()
    assert np.abs(E - ref).max() <= 1e-4 * scale, np.abs(E - ref).max() / scale
    assert np.all(drift < 1e-3 * scale) and np.any(drift > 0)


def test_tensor_core_resync_needs_one_dense_sample(ps):
    c = ps.default_config(N=12, nrep=4, seed=1)
    with pytest.raises(ps.PspinError):
        ps.Engine([c, c], ps.PSPIN_DENSE, ps.make_options(resync_method=ps.RESYNC_TC))
    with pytest.raises(ps.PspinError):
        ps.Engine(c, ps.PSPIN_SPARSE, ps.make_options(resync_method=ps.RESYNC_TC))
