"""The cluster-split sweep (one replica block over 2..16 CTAs exchanging
partial fields through distributed shared memory): every traced move's FP32
dE against the FP64 oracle, and the written-back state against the replay."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfgs(ps, orc, **kw):
    c = ps.default_config(**kw)
    if c.fmc_mode > 0 and c.gamma <= 0.0:
        c.gamma = 0.0 if c.fmc_mode == 1 else 1.0 / (2.0 * (c.N - 1))
    return c, orc.cfg(**kw)


@pytest.mark.parametrize("variant,kw,cluster,warps", [
    (0, dict(N=16, nrep=8, fmc_mode=0, seed=5), 4, 2),
    (0, dict(N=12, nrep=33, fmc_mode=2, seed=7), 2, 4),
    (0, dict(N=24, nrep=16, fmc_mode=0, seed=3, J0=0.5), 16, 2),
    (0, dict(N=20, nrep=8, fmc_mode=0, seed=9), 8, 4),
    (1, dict(N=16, nrep=8, fmc_mode=1, seed=11), 4, 2),
    (0, dict(N=12, nrep=8, fmc_mode=0, seed=2), 4, 1),        # one warp: exchange buffer alignment
    (1, dict(N=16, nrep=8, fmc_mode=1, seed=12), 2, 1),
    (0, dict(N=12, nrep=33, fmc_mode=2, seed=7), -1, 1),      # list-resident one-warp kernel, groups
    (0, dict(N=16, nrep=8, fmc_mode=0, seed=5), -1, 1),       #   ... fully connected tiles
    (1, dict(N=24, nrep=8, fmc_mode=1, seed=13), -1, 1),      #   ... sparse
])
def test_cluster_sweep_dE_against_fp64(ps, orc, variant, kw, cluster, warps):
    c, oc = _cfgs(ps, orc, **kw)
    ref = orc.DenseInit(oc) if variant == 0 else orc.SparseInit(oc)
    nsw, rep = 10, 1
    cap = nsw * (c.N // 2)
    opts = ps.make_options(trace=(0, rep, cap), resync_every=-1, cluster_size=cluster, warps_per_unit=warps)
    with ps.Engine(c, variant, opts) as eng:
        s0 = eng.get_spins()[0][rep].copy()
        eng.fill_betas(1.0 / 0.7)
        eng.sweep(nsw)
        tr = eng.trace(cap)
        s1 = eng.get_spins()[0][rep]
        E, acc, prop = eng.get_results()
    assert len(tr) == cap and 0 < acc[rep] <= prop[rep] == cap
    worst, _, n = orc.check_trace(ref, s0, tr)
    assert worst <= 1e-5, worst
    # replaying the accepted moves gives the state rank 0 wrote back
    s = s0.astype(np.complex64)
    for r in tr:
        if r["accepted"]:
            s[int(r["i0"])] = complex(*r["ai_new"])
            s[int(r["j0"])] = complex(*r["aj_new"])
    np.testing.assert_array_equal(s, s1.astype(np.complex64))


def test_cluster_batch_matches_energy(ps):
    """A batch of uneven samples on clusters of 4: running E equals FP64."""
    cfgs = [ps.default_config(N=N, nrep=40, seed=20 + k, fmc_mode=0) for k, N in enumerate((12, 16, 20))]
    with ps.Engine(cfgs, ps.PSPIN_DENSE, ps.make_options(resync_every=-1, cluster_size=4, warps_per_unit=2)) as eng:
        eng.fill_betas(1.5)
        eng.sweep(30)
        E, acc, prop = eng.get_results()
        e2, e4 = eng.split_energies()
    assert np.all(acc > 0)
    np.testing.assert_allclose(E, e2 + e4, rtol=0, atol=2e-4 * np.abs(e2 + e4).max())


def test_cluster_option_checks(ps):
    c = ps.default_config(N=12, nrep=4, seed=1)
    for bad in (3, 32):
        with pytest.raises(ps.PspinError):
            ps.Engine(c, ps.PSPIN_DENSE, ps.make_options(cluster_size=bad))
    with pytest.raises(ps.PspinError):
        ps.Engine(c, ps.PSPIN_DENSE, ps.make_options(cluster_size=16, warps_per_unit=4))


@pytest.mark.parametrize("variant,kw", [
    (1, dict(N=512, nrep=64, fmc_mode=1, seed=42, gamma=1.0)),     # sparse cube, comb: batches of ~4 moves
    (1, dict(N=64, nrep=40, fmc_mode=2, seed=8, gamma=0.05)),      # sparse, uniform FMC (H2 active: batches of 1)
    (1, dict(N=96, nrep=33, fmc_mode=0, seed=3)),                  # sparse, fully connected selection
    (0, dict(N=12, nrep=33, fmc_mode=2, seed=7)),                  # dense groups (every move conflicts)
])
def test_resident_batched_moves_equal_one_warp(ps, variant, kw):
    """The list-resident kernel with K warps runs batches of consecutive
    moves that commute concurrently; the chain must equal the one-warp
    chain bit for bit (amplitudes, running energies, counters)."""
    c = ps.default_config(**kw)
    if c.fmc_mode == 2 and c.gamma <= 0.0:
        c.gamma = 1.0 / (2.0 * (c.N - 1))
    out = []
    for K in (1, 2, 4, 8):
        with ps.Engine(c, variant, ps.make_options(resync_every=-1, cluster_size=-1, warps_per_unit=K)) as eng:
            eng.fill_betas(1.0 / 0.4)
            eng.sweep(6)
            E, acc, prop = eng.get_results()
            out.append((eng.get_spins()[0], E, acc, prop))
    for K, o in zip((2, 4, 8), out[1:]):
        np.testing.assert_array_equal(o[0], out[0][0], err_msg=f"amplitudes, K={K}")
        for i in (1, 2, 3):
            np.testing.assert_array_equal(o[i], out[0][i], err_msg=f"K={K}")
    assert np.all(out[0][2] > 0)
