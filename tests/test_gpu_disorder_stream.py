"""The streamed sparse set-up (options.disorder_stream = 1).

The reference draws the sparse couplings from one cuRAND call of 2 C(N,4)
normals and keeps the ones at the selected quartets, which needs 45 GB of
device memory at N=512 and more than the device beyond N~700.  The streamed
set-up draws each selected quartet's coupling from its own counter-based
normal instead: the FMC survivors and the partial Fisher-Yates selection are
still the reference's (bit for bit), the couplings follow the same law
(Gaussian, sigma = J4 sqrt(N/n), mean shift as the reference) but are not
its values.  Checked statistically against the bit-exact path at N <= 512,
and run at N=768, where the bit-exact path cannot run on the device.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfg(ps, N, seed, fmc=1, gamma=1.0, T=0.5):
    c = ps.default_config(N=N, nrep=32, seed=seed, fmc_mode=fmc, T=T)
    c.gamma = gamma
    return c


@pytest.mark.parametrize("N,fmc,gamma", [(64, 1, 1.0), (48, 2, 0.05), (512, 1, 1.0)])
def test_streamed_selection_equals_bit_exact(ps, N, fmc, gamma):
    c = _cfg(ps, N, 42, fmc, gamma)
    with ps.Engine(c, ps.PSPIN_SPARSE) as a:
        qa, ga = a.sparse_quartets(0)
        ia = a.info(0)
    with ps.Engine(c, ps.PSPIN_SPARSE, ps.make_options(disorder_stream=True)) as b:
        qb, gb = b.sparse_quartets(0)
        ib = b.info(0)
    np.testing.assert_array_equal(qa, qb)                  # same survivors, same selection
    assert ia.n_quart_active == ib.n_quart_active
    assert not np.array_equal(ga, gb)                      # other coupling values
    # same scale: sigma = J4 sqrt(N / n) with J4 = alpha J = 1 and n = N selected
    sigma = np.sqrt(N / len(ga))
    assert abs(np.std(gb) / sigma - 1.0) < 0.35


def test_streamed_couplings_are_gaussian(ps):
    """Over 24 samples of N=64: mean, variance and kurtosis of the
    normalised couplings as for standard normals."""
    z = []
    for s in range(24):
        c = _cfg(ps, 64, 1000 + s)
        with ps.Engine(c, ps.PSPIN_SPARSE, ps.make_options(disorder_stream=True)) as e:
            _, g = e.sparse_quartets(0)
        z.append(g / np.sqrt(64.0 / len(g)))
    z = np.concatenate(z)
    n = z.size
    assert abs(z.mean()) < 4.0 / np.sqrt(n)
    assert abs(z.var() - 1.0) < 4.0 * np.sqrt(2.0 / n)
    k = np.mean(z ** 4) / z.var() ** 2
    assert abs(k - 3.0) < 4.0 * np.sqrt(24.0 / n)


def test_streamed_energy_statistics_match_bit_exact(ps):
    """Disorder-averaged <E>/N after 300 sweeps at T=0.5 over 16 samples of
    N=64 (comb FMC): the two coupling sources agree within 3.5 sigma."""
    out = {}
    for stream in (False, True):
        cfgs = [_cfg(ps, 64, 200 + s) for s in range(16)]
        with ps.Engine(cfgs, ps.PSPIN_SPARSE, ps.make_options(disorder_stream=stream)) as e:
            e.fill_betas(2.0)
            e.sweep(300)
            E, _, _ = e.get_results()
        per = E.reshape(16, 32).mean(axis=1) / 64
        out[stream] = (per.mean(), per.std(ddof=1) / np.sqrt(16))
    z = (out[True][0] - out[False][0]) / np.hypot(out[True][1], out[False][1])
    print(f"<E>/N bit-exact {out[False][0]:.4f}+-{out[False][1]:.4f}  streamed {out[True][0]:.4f}+-{out[True][1]:.4f}"
          f"  z={z:.2f}")
    assert abs(z) < 3.5


def test_streamed_setup_beyond_device_memory(ps):
    """N=768: the bit-exact path would need 2 C(768,4) doubles (226 GB);
    the streamed set-up builds the sample and sweeps it (cube constraint kept,
    running energy equal to the FP64 recompute)."""
    c = _cfg(ps, 768, 7)
    c.nrep = 32
    with ps.Engine(c, ps.PSPIN_SPARSE, ps.make_options(disorder_stream=True, resync_every=-1)) as e:
        info = e.info(0)
        assert info.n_quartets == 768 and info.n_quart_active > 768
        # the reference's cube initialisation sums |a|^4 over a tree that
        # drops terms for N not a power of two, so each replica starts at its
        # own constraint value; the moves keep it
        s0 = np.sum(np.abs(e.get_spins()[0].astype(np.complex128)) ** 4, axis=1)
        e.fill_betas(2.0)
        e.sweep(20)
        sp = e.get_spins()[0]
        E, acc, _ = e.get_results()
        e2, e4 = e.split_energies()
    assert np.all(acc > 0)
    np.testing.assert_allclose(np.sum(np.abs(sp.astype(np.complex128)) ** 4, axis=1), s0, rtol=1e-4)
    np.testing.assert_allclose(E, e2 + e4, rtol=0, atol=1e-3 * np.abs(e2 + e4).max())
