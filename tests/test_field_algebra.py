"""CPU check of the algebra the sweep kernel is built on.

For member m of a quartet with partner p and opposite pair {o1,o2} (channel
classes of disorder.h:9-16), the quartet's energy term is
-Re[a_m * g a_p conj(a_o1) conj(a_o2)], so with
    h_m = sum_{q containing m} g a_p conj(a_o1 a_o2) + sum_{j != m} g2_mj conj(a_j)
a pair move (i,j) changes the energy by exactly
    dE = -Re[(a_i'-a_i) h_i(a_j')] - Re[(a_j'-a_j) h_j(a_i)].
Checked here in FP64 numpy against the oracle's full-energy differences
(the reference's chain form, mc.cu:323-405) on random moves, dense and sparse.
"""
import numpy as np
import pytest

U = {0: (0, 1), 1: (0, 3), 2: (0, 2)}
C = {0: (2, 3), 1: (1, 2), 2: (1, 3)}


def site_records(quartets):
    """quartets: iterable of (i,j,k,l,ch,g) -> per-site list of (p,o1,o2,g)."""
    rec = {}
    for (i, j, k, l, ch, g) in quartets:
        q = (i, j, k, l)
        for pos in range(4):
            mine, opp = (U[ch], C[ch]) if pos in U[ch] else (C[ch], U[ch])
            p = q[mine[1] if mine[0] == pos else mine[0]]
            o1, o2 = sorted((q[opp[0]], q[opp[1]]))
            rec.setdefault(q[pos], []).append((p, o1, o2, g))
    return rec


def field(rec, g2, h2_active, a, m):
    h = 0j
    for (p, o1, o2, g) in rec.get(m, []):
        h += g * a[p] * np.conj(a[o1]) * np.conj(a[o2])
    if h2_active:
        N = len(a)
        for j in range(N):
            if j != m:
                h += g2[m, j] * np.conj(a[j])
    return h


def dense_quartets(ref):
    N = ref.N
    g4 = ref.g4[0::2]
    out, q = [], 0
    for l in range(3, N):
        for k in range(2, l):
            for j in range(1, k):
                for i in range(j):
                    m = ref.mask[q]
                    if m and g4[q] != 0.0:
                        for ch in range(3):
                            if m & (1 << ch):
                                out.append((i, j, k, l, ch, g4[q]))
                    q += 1
    return out


@pytest.mark.parametrize("N,fmc,seed", [(8, 0, 1), (10, 2, 3), (11, 1, 4), (12, 2, 42)])
def test_dense_field_decomposition(orc, N, fmc, seed):
    ref = orc.DenseInit(orc.cfg(N=N, nrep=2, fmc_mode=fmc, seed=seed, gamma=0.3 if fmc == 2 else 0.0))
    rec = site_records(dense_quartets(ref))
    g2 = ref.g2.reshape(N, N, 2)[..., 0]
    h2 = ref.info.h2_active
    rng = np.random.default_rng(seed)
    a = ref.spins_c()[0].copy()
    # energy identity: E4 = -1/4 sum Re[a_m h4_m], E2 = -1/2 sum Re[a_m h2_m]
    e2, e4 = ref.energy(a)
    h4 = [field(rec, g2, 0, a, m) for m in range(N)]
    assert abs(e4 + 0.25 * sum((a[m] * h4[m]).real for m in range(N))) < 1e-10 * (1 + abs(e4))
    for _ in range(25):
        i, j = sorted(rng.choice(N, 2, replace=False))
        new = a.copy()
        new[i] = a[i] * np.exp(1j * rng.uniform(0, 6.3)) * rng.uniform(0.2, 1.5)
        new[j] = a[j] * np.exp(1j * rng.uniform(0, 6.3)) * rng.uniform(0.2, 1.5)
        with_aj_new = a.copy()
        with_aj_new[j] = new[j]
        hi = field(rec, g2, h2, with_aj_new, i)
        hj = field(rec, g2, h2, a, j)
        dE = -((new[i] - a[i]) * hi).real - ((new[j] - a[j]) * hj).real
        d64 = sum(ref.energy(new)) - sum(ref.energy(a))
        assert abs(dE - d64) < 1e-11 * (1 + abs(d64) + ref.abs_terms(a, new, i, j))
        if rng.uniform() < 0.5:
            a = new


@pytest.mark.parametrize("N,fmc,seed", [(10, 0, 5), (16, 2, 7)])
def test_sparse_field_decomposition(orc, N, fmc, seed):
    ref = orc.SparseInit(orc.cfg(N=N, nrep=1, fmc_mode=fmc, seed=seed, gamma=0.2 if fmc == 2 else 0.0))
    qs = [tuple(int(x) for x in ref.q[t]) + (ref.qg[t],) for t in range(len(ref.qg))]
    rec = site_records(qs)
    g2 = ref.g2.reshape(N, N, 2)[..., 0]
    rng = np.random.default_rng(seed)
    a = ref.spins_c()[0].copy()
    for _ in range(40):
        i, j = sorted(rng.choice(N, 2, replace=False))
        new = a.copy()
        new[i] = rng.normal() + 1j * rng.normal()
        new[j] = rng.normal() + 1j * rng.normal()
        w = a.copy()
        w[j] = new[j]
        dE = -((new[i] - a[i]) * field(rec, g2, ref.info.h2_active, w, i)).real \
             - ((new[j] - a[j]) * field(rec, g2, ref.info.h2_active, a, j)).real
        d64 = sum(ref.energy(new)) - sum(ref.energy(a))
        assert abs(dE - d64) < 1e-11 * (1 + abs(d64))
        a = new
