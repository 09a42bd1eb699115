"""Per-move dE against the FP64 oracle at the sizes and on the kernel shapes
the benchmark configurations run.

  * large dense MC (N=128, fully connected, 64 replicas at T=0.5) on the
    cluster split the autotuner picks there: 16 CTAs x 2 warps per replica
    block (and 8 x 4);
  * the batched benchmark's shape (2 CTAs x 4 warps per replica block,
    fully connected tiles, 96 replicas) at N=48 and N=64, and N=24/32 for
    the other classes of its N mix;
  * sparse cube PT at N=512 (comb FMC, gamma=1, N quartets picked by the
    partial Fisher-Yates) on the list-resident kernel it runs on, with one
    warp and with 8 warps running batches of commuting moves, and on the
    ring-fed kernels.

Every traced move's FP32 dE must be within 1e-5 of sum|terms| of the FP64
difference of full chain-form energies on the same FP32 amplitudes; the
plain relative error |dE32 - dE64| / |dE64| and the hamiltonian.cu-form
difference (the g2 diagonal, which that form keeps and the chain does not)
are printed beside it.  Replaying the accepted moves must give the
amplitudes the kernel wrote back, bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _replay(s0, tr):
    s = s0.astype(np.complex64)
    for r in tr:
        if r["accepted"]:
            s[int(r["i0"])] = complex(*r["ai_new"])
            s[int(r["j0"])] = complex(*r["aj_new"])
    return s


def _run(ps, cfg, variant, cluster, warps, nsweeps, rep, T):
    cap = nsweeps * (cfg.N // 2)
    opts = ps.make_options(trace=(0, rep, cap), resync_every=-1, cluster_size=cluster, warps_per_unit=warps)
    with ps.Engine(cfg, variant, opts) as eng:
        s0 = eng.get_spins()[0][rep].copy()
        eng.fill_betas(1.0 / T)
        eng.sweep(nsweeps)
        tr = eng.trace(cap)
        s1 = eng.get_spins()[0][rep]
        E, acc, prop = eng.get_results()
        extra = None
        if variant == ps.PSPIN_SPARSE:
            extra = eng.sparse_quartets(0), eng.info(0)
    assert len(tr) == cap and prop[rep] == cap
    assert 0 < acc[rep] == int(tr["accepted"].sum())
    return s0, s1, tr, extra


@pytest.mark.parametrize("cluster,warps", [(16, 2), (8, 4)])
def test_large_dense_n128_cluster_per_move(ps, orc, cluster, warps):
    """Large dense MC: N=128 FC, 64 replicas at T=0.5 (two replica blocks)."""
    kw = dict(N=128, nrep=64, fmc_mode=0, seed=4242, T=0.5)
    cfg = ps.default_config(**kw)
    ref = orc.DenseInit(orc.cfg(**kw))
    s0, s1, tr, _ = _run(ps, cfg, ps.PSPIN_DENSE, cluster, warps, nsweeps=2, rep=37, T=0.5)
    rep = {}
    worst, rel, n = orc.check_trace(ref, s0, tr, report=rep)
    print(f"N=128 FC, {cluster} CTAs x {warps} warps: {n} moves, max err/sum|terms| {worst:.2e}, "
          f"plain relative max {rel:.2e} median {rep['rel_median']:.2e}, "
          f"hamiltonian.cu-form diagonal term up to {rep['diag_max']:.2e} of sum|terms| "
          f"(dE32 + diagonal vs that form: {rep['ham_err_max']:.2e})")
    assert worst <= TOL, worst
    assert rep["ham_err_max"] <= TOL
    np.testing.assert_array_equal(_replay(s0, tr), s1.astype(np.complex64))


@pytest.mark.parametrize("N", [24, 32, 48, 64])
def test_benchmark_shape_per_move(ps, orc, N):
    """The batched benchmark's kernel: 2 CTAs x 4 warps per replica block on
    fully connected tiles, 96 replicas (24 temperatures x 4) per sample."""
    kw = dict(N=N, nrep=96, fmc_mode=0, seed=1000 + N, T=0.4)
    cfg = ps.default_config(**kw)
    ref = orc.DenseInit(orc.cfg(**kw))
    s0, s1, tr, _ = _run(ps, cfg, ps.PSPIN_DENSE, 2, 4, nsweeps=3 if N >= 48 else 8, rep=70, T=0.4)
    rep = {}
    worst, rel, n = orc.check_trace(ref, s0, tr, report=rep)
    print(f"N={N} FC, 2 CTAs x 4 warps: {n} moves, max err/sum|terms| {worst:.2e}, plain relative max {rel:.2e} "
          f"median {rep['rel_median']:.2e}, diagonal term up to {rep['diag_max']:.2e}")
    assert worst <= TOL, worst
    assert rep["ham_err_max"] <= TOL
    np.testing.assert_array_equal(_replay(s0, tr), s1.astype(np.complex64))


@pytest.mark.parametrize("cluster,warps", [(-1, 1), (-1, 8), (1, 4), (4, 2)])
def test_sparse_n512_comb_per_move(ps, orc, cluster, warps):
    """Sparse cube PT: N=512, comb FMC, gamma=1, 128 replicas at T=0.3.  The
    oracle's set-up at this size needs 2 C(512,4) host normals (45 GB), so
    the replay uses the engine's quartet list, whose selection and couplings
    equal the reference's bit for bit (tests/test_golden.py,
    sparse_n512_fmc1_s42)."""
    cfg = ps.default_config(N=512, nrep=128, fmc_mode=1, seed=42, T=0.3)
    cfg.gamma = 1.0
    s0, s1, tr, ((q, g), info) = _run(ps, cfg, ps.PSPIN_SPARSE, cluster, warps, nsweeps=4, rep=99, T=0.3)
    assert info.h2_active == 0 and len(g) == 512
    ref = orc.SparseFromList(512, q, g)
    rep = {}
    worst, rel, n = orc.check_trace(ref, s0, tr, report=rep)
    print(f"N=512 sparse comb, shape ({cluster},{warps}): {n} moves, max err/sum|terms| {worst:.2e}, "
          f"plain relative max {rel:.2e} median {rep['rel_median']:.2e}")
    assert worst <= TOL, worst
    np.testing.assert_array_equal(_replay(s0, tr), s1.astype(np.complex64))
    # cube constraint kept by every move (spins_sparse.h:26-56)
    assert abs(np.sum(np.abs(s1.astype(np.complex128)) ** 4) - 512.0) < 5e-2
