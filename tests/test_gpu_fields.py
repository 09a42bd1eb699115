"""All-site local fields: the tensor-core split-BF16 contraction against FP64.

pspin_local_fields(FIELDS_TC_BF16X3) forms pair products, splits them and the
pair-space couplings into BF16 hi+lo parts and contracts them on the sm100
tensor cores with FP32 accumulation; FIELDS_FP64 sums the quartet table in
FP64.  The FP64 fields are checked against an independent numpy evaluation
of the field definition on the oracle's couplings; the tensor-core fields and
energies against the FP64 ones (error stated relative to the largest field /
per site for the energy).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _numpy_fields(ref, a):
    from tests.test_field_algebra import dense_quartets, field, site_records
    rec = site_records(dense_quartets(ref))
    N = ref.N
    g2 = ref.g2.reshape(N, N, 2)[..., 0]
    return np.array([field(rec, g2, ref.info.h2_active, a, m) for m in range(N)])


@pytest.mark.parametrize("kw", [dict(N=10, nrep=4, fmc_mode=0, seed=3), dict(N=12, nrep=2, fmc_mode=2, seed=7)])
def test_fp64_fields_match_definition(ps, orc, kw):
    c = ps.default_config(**kw)
    if c.fmc_mode == 2:
        c.gamma = 1.0 / (2.0 * (c.N - 1))
    ref = orc.DenseInit(orc.cfg(**kw))
    with ps.Engine(c) as eng:
        h, E = eng.local_fields(0, ps.FIELDS_FP64)
        sp = eng.get_spins()[0]
        for r in range(c.nrep):
            hn = _numpy_fields(ref, sp[r])
            np.testing.assert_allclose(h[r], hn, rtol=0, atol=1e-10 * max(1.0, np.abs(hn).max()))
            assert abs(E[r] - sum(ref.energy(sp[r]))) < 1e-9 * c.N


@pytest.mark.parametrize("kw", [dict(N=16, nrep=8, fmc_mode=0, seed=1),
                                dict(N=32, nrep=6, fmc_mode=2, seed=42, gamma=0.1),
                                dict(N=64, nrep=12, fmc_mode=0, seed=5),
                                dict(N=128, nrep=8, fmc_mode=0, seed=9)])
def test_tensor_core_fields_match_fp64(ps, kw):
    c = ps.default_config(**kw)
    with ps.Engine(c) as eng:
        eng.fill_betas(2.0)
        eng.sweep(4)
        h64, e64 = eng.local_fields(0, ps.FIELDS_FP64)
        htc, etc = eng.local_fields(0, ps.FIELDS_TC_BF16X3)
        rel = np.abs(htc - h64).max() / np.abs(h64).max()
        de = np.abs(etc - e64).max() / c.N
        print(f"N={c.N}: max field error {rel:.2e} of max|h|, energy error {de:.2e} per site")
        assert rel < 1e-4
        assert de < 1e-4
        # a second call reuses the pair-space couplings
        htc2, _ = eng.local_fields(0, ps.FIELDS_TC_BF16X3)
        assert np.array_equal(htc, htc2)
