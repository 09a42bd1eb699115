"""The plain sweep with 2 or 3 replicas per lane (one block = 64 or 96
replicas of a sample; every staged coupling serves all of them).

The per-replica summation order is the one of the one-replica-per-lane
kernels of the same block shape, so the chain must be the same bit for bit:
amplitudes, running energies and move counters, single-temperature sweeps
and PT runs (exchange + graph replay) alike, ragged last blocks included.
Traced moves of a replica in the third slot are checked against the FP64
oracle, as for every other sweep kernel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfg(ps, **kw):
    c = ps.default_config(**kw)
    if c.fmc_mode == 2 and c.gamma <= 0.0:
        c.gamma = 1.0 / (2.0 * (c.N - 1))
    return c


def _run(ps, cfgs, variant, K, cluster, warps, nsw=6, beta=1.0 / 0.5):
    opts = ps.make_options(resync_every=-1, cluster_size=cluster, warps_per_unit=warps, replicas_per_lane=K)
    with ps.Engine(cfgs, variant, opts) as eng:
        eng.fill_betas(beta)
        eng.sweep(nsw)
        E, acc, prop = eng.get_results()
        return eng.get_spins(), E, acc, prop


@pytest.mark.parametrize("variant,kws,cluster,warps", [
    (0, [dict(N=16, nrep=100, fmc_mode=0, seed=5)], 1, 4),                        # tiles, CTA kernel, ragged 4
    (0, [dict(N=12, nrep=70, fmc_mode=2, seed=7)], 2, 4),                         # groups, cluster 2
    (0, [dict(N=24, nrep=96, fmc_mode=0, seed=3, J0=0.5)], 16, 2),                # cluster 16
    (0, [dict(N=20, nrep=40, fmc_mode=0, seed=9)], 4, 1),                         # one warp per CTA
    (1, [dict(N=32, nrep=97, fmc_mode=1, seed=11, gamma=1.0)], 4, 2),             # sparse cube
    (1, [dict(N=24, nrep=64, fmc_mode=2, seed=12, gamma=0.05)], 1, 8),            # sparse sphere, H2 on
    (0, [dict(N=N, nrep=R, fmc_mode=0, seed=30 + k)                               # uneven batch
         for k, (N, R) in enumerate(((24, 96), (32, 33), (48, 130), (16, 1)))], 2, 4),
])
def test_replicas_per_lane_equal_one(ps, variant, kws, cluster, warps):
    cfgs = [_cfg(ps, **kw) for kw in kws]
    base = _run(ps, cfgs, variant, 1, cluster, warps)
    assert np.all(base[2][base[3] > 0] >= 0) and base[2].sum() > 0
    for K in (2, 3):
        got = _run(ps, cfgs, variant, K, cluster, warps)
        for a, b in zip(got[0], base[0]):
            np.testing.assert_array_equal(a, b, err_msg=f"amplitudes, K={K}")
        for i in (1, 2, 3):
            np.testing.assert_array_equal(got[i], base[i], err_msg=f"K={K}")


def test_replicas_per_lane_pt_equal_one(ps):
    """PT with the device exchange and the captured step graph."""
    NT, nr = 24, 4
    cfgs = [ps.default_config(N=N, nrep=NT * nr, seed=40 + k, fmc_mode=0) for k, N in enumerate((24, 32, 48))]
    T, beta = ps.temperature_schedule(NT, 0.2, 1.6, True)
    out = []
    for K in (1, 3):
        opts = ps.make_options(resync_every=64, cluster_size=2, warps_per_unit=4, replicas_per_lane=K)
        with ps.Engine(cfgs, ps.PSPIN_DENSE, opts) as eng:
            eng.pt_init(NT, nr, beta, 1)
            eng.pt_run(80)
            E, acc, prop = eng.get_results()
            out.append((eng.get_spins(), E, acc, prop, [eng.pt_get(k) for k in range(len(cfgs))]))
    for a, b in zip(out[1][0], out[0][0]):
        np.testing.assert_array_equal(a, b)
    for i in (1, 2, 3):
        np.testing.assert_array_equal(out[1][i], out[0][i])
    for pa, pb in zip(out[1][4], out[0][4]):
        for x, y in zip(pa, pb):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("variant,kw,cluster,warps,rep", [
    (0, dict(N=16, nrep=96, fmc_mode=0, seed=5), 2, 4, 70),
    (0, dict(N=12, nrep=80, fmc_mode=2, seed=7), 1, 2, 77),
    (1, dict(N=24, nrep=96, fmc_mode=1, seed=13, gamma=1.0), 4, 2, 95),
])
def test_replicas_per_lane_dE_against_fp64(ps, orc, variant, kw, cluster, warps, rep):
    c = _cfg(ps, **kw)
    oc = orc.cfg(**kw)
    ref = orc.DenseInit(oc) if variant == 0 else orc.SparseInit(oc)
    nsw = 10
    cap = nsw * (c.N // 2)
    opts = ps.make_options(trace=(0, rep, cap), resync_every=-1, cluster_size=cluster, warps_per_unit=warps,
                           replicas_per_lane=3)
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
    s = s0.astype(np.complex64)
    for r in tr:
        if r["accepted"]:
            s[int(r["i0"])] = complex(*r["ai_new"])
            s[int(r["j0"])] = complex(*r["aj_new"])
    np.testing.assert_array_equal(s, s1.astype(np.complex64))


def test_replicas_per_lane_option_checks(ps):
    c = ps.default_config(N=12, nrep=8, seed=1)
    for bad in (-1, 4):
        with pytest.raises(ps.PspinError):
            ps.Engine(c, ps.PSPIN_DENSE, ps.make_options(replicas_per_lane=bad))
    with pytest.raises(ps.PspinError):      # 96 replicas x N=320 amplitudes do not fit a CTA
        ps.Engine(ps.default_config(N=320, nrep=8, seed=1, fmc_mode=1, gamma=1.0), ps.PSPIN_SPARSE,
                  ps.make_options(replicas_per_lane=3, cluster_size=1, warps_per_unit=1, disorder_stream=True))


def test_autotune_lanes(ps):
    cfgs = [ps.default_config(N=N, nrep=96, seed=50 + k, fmc_mode=0) for k, N in enumerate((24, 32))]
    with ps.Engine(cfgs, ps.PSPIN_DENSE, ps.make_options(resync_every=-1)) as eng:
        eng.fill_betas(2.0)
        eng.sweep(2)
        s_before = [x.copy() for x in eng.get_spins()]
        E_before = eng.get_results()[0].copy()
        w, cl, K, ms = eng.autotune_lanes(sweeps=2)
        assert K in (1, 2, 3) and w in (1, 2, 4, 8) and cl in (0, 1, 2, 4, 8, 16)
        assert ms.shape == (3, 6, 4)
        assert np.all(ms[1:, 0, :] == -1)          # the resident kernel has one replica per lane
        assert (ms[1:] > 0).any() and (ms[0] > 0).any()
        best = ms[K - 1, [0, 1, 2, 4, 8, 16].index(cl), [1, 2, 4, 8].index(w)]
        assert best > 0 and best <= ms[ms > 0].min() + 1e-6
        # the trials leave the chain where it was
        for a, b in zip(eng.get_spins(), s_before):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(eng.get_results()[0], E_before)
