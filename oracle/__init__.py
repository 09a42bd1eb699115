"""ctypes face of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline / reference legs.  The product
(cuda_pspin_b200, libpspin.so, the drivers) never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
REF_DIR = os.path.join(_HERE, "_ref")

_lib = None


class OrcConfig(ctypes.Structure):
    _fields_ = [("save_freq", ctypes.c_int), ("verbose", ctypes.c_int), ("N", ctypes.c_int),
                ("nrep", ctypes.c_int), ("T", ctypes.c_double), ("J", ctypes.c_double),
                ("J0", ctypes.c_double), ("alpha", ctypes.c_double), ("alpha0", ctypes.c_double),
                ("mc_iterations", ctypes.c_int), ("seed", ctypes.c_uint64), ("label", ctypes.c_int),
                ("dev", ctypes.c_int), ("fmc_mode", ctypes.c_int), ("gamma", ctypes.c_double)]


class OrcInfo(ctypes.Structure):
    _fields_ = [("n_pairs_active", ctypes.c_int64), ("n_quart_active", ctypes.c_int64),
                ("h2_active", ctypes.c_int), ("n_sparse", ctypes.c_int)]


class OrcSweepArgs(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int), ("N", ctypes.c_int), ("nrep", ctypes.c_int),
                ("h2_active", ctypes.c_int), ("g2", ctypes.c_void_p), ("g4", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("nq", ctypes.c_int), ("q_ijklch", ctypes.c_void_p),
                ("q_g", ctypes.c_void_p), ("spins", ctypes.c_void_p), ("energies", ctypes.c_void_p),
                ("betas", ctypes.c_void_p), ("accepted", ctypes.c_void_p), ("proposed", ctypes.c_void_p),
                ("seeds", ctypes.c_void_p), ("move_counter", ctypes.c_void_p), ("nthreads", ctypes.c_int)]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        i64, u64, vp, d, i32 = ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        for name, res, args in [
            ("orc_n_quartets", i64, [i32]), ("orc_encode_quartet", i64, [i32, i32, i32, i32]),
            ("orc_decode_quartet", None, [i64, vp, vp, vp, vp]),
            ("orc_three_type", i64, [i32, i32, i32, vp]),
            ("orc_auto_gamma", d, [i32, i32, d]),
            ("orc_temperature_schedule", None, [i32, d, d, i32, vp, vp]),
            ("orc_omega", None, [i32, i32, u64, vp]),
            ("orc_fmc_g4_mask", None, [vp, i32, vp, d]),
            ("orc_fmc_channel", ctypes.c_uint8, [i32, i32, i32, i32, vp, d]),
            ("orc_count_active_g4", i64, [vp, i64]),
            ("orc_count_survivors", i64, [i32, vp, d, vp]),
            ("orc_curand_normals", i32, [u64, i64, vp]),
            ("orc_init_dense", i32, [ctypes.POINTER(OrcConfig), i32, vp, vp, vp, vp, vp, vp, ctypes.POINTER(OrcInfo)]),
            ("orc_init_sparse", i32, [ctypes.POINTER(OrcConfig), i32, vp, vp, vp, vp, vp, vp, ctypes.POINTER(OrcInfo)]),
            ("orc_sparse_select", i32, [i32, vp, d, i32, u64, i32, vp, vp]),
            ("orc_partial_shuffle", None, [vp, i64, i32, u64]),
            ("orc_normalize_sphere", None, [vp, i32, i32]), ("orc_normalize_cube", None, [vp, i32, i32]),
            ("orc_energy_dense", None, [i32, vp, vp, vp, i32, vp, vp, vp]),
            ("orc_energy_sparse", None, [i32, vp, i32, vp, vp, i32, vp, vp, vp]),
            ("orc_energy_h2_with_diag", d, [i32, vp, vp]),
            ("orc_dense_abs_terms", d, [i32, vp, vp, vp, i32, vp, vp, i32, i32]),
            ("orc_sparse_abs_terms", d, [i32, vp, i32, vp, vp, i32, vp, vp, i32, i32]),
            ("orc_propose_sphere", None, [vp, vp, d, d, d, vp, vp]),
            ("orc_propose_cube", None, [vp, vp, d, d, d, vp, vp]),
            ("orc_philox4x32_10", None, [vp, vp, vp]),
            ("orc_srand48_state", u64, [ctypes.c_long]), ("orc_drand48", d, [vp]),
            ("orc_exchange", None, [i32, i32, vp, vp, vp, vp, vp, vp, vp]),
            ("orc_sweep", None, [ctypes.POINTER(OrcSweepArgs), i32]),
            ("orc_splitmix64", u64, [vp]), ("orc_replica_seeds", None, [u64, i32, vp]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def P(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def n_quartets(N: int) -> int:
    return N * (N - 1) * (N - 2) * (N - 3) // 24


def cfg(**kw) -> OrcConfig:
    c = OrcConfig(save_freq=100, verbose=0, N=64, nrep=1, T=1.0, J=2.0, J0=0.0, alpha=0.5, alpha0=0.5,
                  mc_iterations=10000, seed=42, label=-1, dev=-1, fmc_mode=0, gamma=0.0)
    for k, v in kw.items():
        setattr(c, k, v)
    if c.fmc_mode > 0 and c.gamma <= 0.0:
        c.gamma = lib().orc_auto_gamma(c.fmc_mode, c.N, c.gamma)
    return c


def omega(N: int, fmc_mode: int, seed: int) -> np.ndarray:
    w = np.zeros(N)
    lib().orc_omega(N, fmc_mode, seed, P(w))
    return w


def fmc_mask(N: int, w: np.ndarray, gamma: float) -> np.ndarray:
    m = np.zeros(n_quartets(N), np.uint8)
    wc = np.ascontiguousarray(w, np.float64)
    lib().orc_fmc_g4_mask(P(m), N, P(wc), gamma)
    return m


def curand_normals(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count)
    rc = lib().orc_curand_normals(seed, count, P(out))
    if rc:
        raise RuntimeError(f"cuRAND host generator failed ({rc})")
    return out


class DenseInit:
    """mc_init (mc.cu:411-562) on the CPU."""

    def __init__(self, c: OrcConfig, init_exact: bool = False):
        N, R = c.N, c.nrep
        nq = n_quartets(N)
        self.cfg = c
        self.N, self.R = N, R
        self.g2 = np.zeros(2 * N * N)
        self.g4 = np.zeros(2 * nq)
        self.mask = np.zeros(nq, np.uint8)
        self.omega = np.zeros(N)
        self.spins = np.zeros(2 * N * R)
        self.energies = np.zeros(R)
        self.info = OrcInfo()
        rc = lib().orc_init_dense(ctypes.byref(c), int(init_exact), P(self.g2), P(self.g4), P(self.mask),
                                  P(self.omega), P(self.spins), P(self.energies), ctypes.byref(self.info))
        if rc:
            raise RuntimeError("oracle dense init failed")

    def spins_c(self) -> np.ndarray:
        v = self.spins.reshape(self.R, self.N, 2)
        return v[..., 0] + 1j * v[..., 1]

    def energy(self, spins_c: np.ndarray):
        """(E2, E4) of one replica given complex amplitudes."""
        s = np.ascontiguousarray(np.stack([spins_c.real, spins_c.imag], -1).ravel())
        e2, e4 = ctypes.c_double(), ctypes.c_double()
        lib().orc_energy_dense(self.N, P(self.g2), P(self.g4), P(self.mask), self.info.h2_active, P(s),
                               ctypes.byref(e2), ctypes.byref(e4))
        return e2.value, e4.value

    def abs_terms(self, old_c: np.ndarray, new_c: np.ndarray, i0: int, j0: int) -> float:
        so = np.ascontiguousarray(np.stack([old_c.real, old_c.imag], -1).ravel())
        sn = np.ascontiguousarray(np.stack([new_c.real, new_c.imag], -1).ravel())
        return lib().orc_dense_abs_terms(self.N, P(self.g2), P(self.g4), P(self.mask), self.info.h2_active,
                                         P(so), P(sn), i0, j0)


class SparseInit:
    """mc_sparse_init (mc_sparse.cu:390-604) on the CPU (small N)."""

    def __init__(self, c: OrcConfig, init_exact: bool = False):
        N, R = c.N, c.nrep
        self.cfg = c
        self.N, self.R = N, R
        self.g2 = np.zeros(2 * N * N)
        self.q = np.zeros(5 * N, np.int32)
        self.qg = np.zeros(N)
        self.omega = np.zeros(N)
        self.spins = np.zeros(2 * N * R)
        self.energies = np.zeros(R)
        self.info = OrcInfo()
        rc = lib().orc_init_sparse(ctypes.byref(c), int(init_exact), P(self.g2), P(self.q), P(self.qg),
                                   P(self.omega), P(self.spins), P(self.energies), ctypes.byref(self.info))
        if rc:
            raise RuntimeError("oracle sparse init failed")
        ns = self.info.n_sparse
        self.q = self.q[:5 * ns].reshape(ns, 5)
        self.qg = self.qg[:ns]

    def spins_c(self) -> np.ndarray:
        v = self.spins.reshape(self.R, self.N, 2)
        return v[..., 0] + 1j * v[..., 1]

    def energy(self, spins_c: np.ndarray):
        s = np.ascontiguousarray(np.stack([spins_c.real, spins_c.imag], -1).ravel())
        q = np.ascontiguousarray(self.q.ravel())
        e2, e4 = ctypes.c_double(), ctypes.c_double()
        lib().orc_energy_sparse(self.N, P(self.g2), len(self.qg), P(q), P(self.qg), self.info.h2_active, P(s),
                                ctypes.byref(e2), ctypes.byref(e4))
        return e2.value, e4.value

    def abs_terms(self, old_c, new_c, i0, j0) -> float:
        so = np.ascontiguousarray(np.stack([old_c.real, old_c.imag], -1).ravel())
        sn = np.ascontiguousarray(np.stack([new_c.real, new_c.imag], -1).ravel())
        q = np.ascontiguousarray(self.q.ravel())
        return lib().orc_sparse_abs_terms(self.N, P(self.g2), len(self.qg), P(q), P(self.qg),
                                          self.info.h2_active, P(so), P(sn), i0, j0)


class SparseFromList:
    """The sparse chain's energy (mc_sparse.cu:258-315) over a given quartet
    list: for replaying traces at sizes whose oracle set-up (2*C(N,4) host
    normals) is too large, with the list and couplings taken from a run that
    is itself checked bit for bit against the reference's selection."""

    def __init__(self, N: int, q: np.ndarray, qg: np.ndarray, g2_real: np.ndarray | None = None,
                 h2_active: int = 0):
        self.N = N
        self.q = np.ascontiguousarray(q, np.int32).reshape(-1, 5)
        self.qg = np.ascontiguousarray(qg, np.float64)
        g2 = np.zeros((N, N, 2))
        if g2_real is not None:
            g2[..., 0] = g2_real
        self.g2 = np.ascontiguousarray(g2.ravel())
        self.h2 = int(h2_active)

    def energy(self, spins_c: np.ndarray):
        s = np.ascontiguousarray(np.stack([spins_c.real, spins_c.imag], -1).ravel())
        q = np.ascontiguousarray(self.q.ravel())
        e2, e4 = ctypes.c_double(), ctypes.c_double()
        lib().orc_energy_sparse(self.N, P(self.g2), len(self.qg), P(q), P(self.qg), self.h2, P(s),
                                ctypes.byref(e2), ctypes.byref(e4))
        return e2.value, e4.value

    def abs_terms(self, old_c, new_c, i0, j0) -> float:
        so = np.ascontiguousarray(np.stack([old_c.real, old_c.imag], -1).ravel())
        sn = np.ascontiguousarray(np.stack([new_c.real, new_c.imag], -1).ravel())
        q = np.ascontiguousarray(self.q.ravel())
        return lib().orc_sparse_abs_terms(self.N, P(self.g2), len(self.qg), P(q), P(self.qg), self.h2,
                                          P(so), P(sn), i0, j0)


def check_trace(ref, spins0: np.ndarray, trace: np.ndarray, tol: float = 1e-5, report: dict | None = None):
    """Replays a traced replica move by move.  For every move the FP32 dE the
    kernel decided on is compared with the FP64 difference of full energies
    (the chain's form, g2 over i<j) on the same FP32-stored amplitudes.
    Returns (max |dE32-dE64| / sum|terms|, max plain relative error
    |dE32-dE64| / |dE64|, n_moves).

    When `report` is a dict it also receives the plain relative error's
    median and the hamiltonian.cu form (hamiltonian.cu:30-38, g2 over i<=j):
    the largest diagonal change |g_ii d|a_i|^2 + g_jj d|a_j|^2| of a move
    relative to sum|terms| ("diag_max"), i.e. how far that form's dE is from
    the chain's, and the largest error of dE32 + that diagonal change against
    the FP64 difference of hamiltonian.cu-form energies ("ham_err_max")."""
    s = np.array(spins0, np.complex128)
    worst, worst_rel = 0.0, 0.0
    rels, diag_max, ham_err = [], 0.0, 0.0
    e_cur = None                   # energies of the current state (the last move's old or new)
    g2d = None
    if report is not None and isinstance(ref, DenseInit):
        N = len(s)
        g2c = np.ascontiguousarray(ref.g2, np.float64)
        g2d = g2c.reshape(N, N, 2)[np.arange(N), np.arange(N), 0]
    for rec in trace:
        i0, j0 = int(rec["i0"]), int(rec["j0"])
        ai_old = complex(rec["ai_old"][0], rec["ai_old"][1])
        aj_old = complex(rec["aj_old"][0], rec["aj_old"][1])
        if s[i0] != ai_old or s[j0] != aj_old:
            raise AssertionError(f"replay diverged at move ({i0},{j0})")
        new = s.copy()
        new[i0] = complex(rec["ai_new"][0], rec["ai_new"][1])
        new[j0] = complex(rec["aj_new"][0], rec["aj_new"][1])
        e2o, e4o = e_cur if e_cur is not None else ref.energy(s)
        e2n, e4n = ref.energy(new)
        d64 = (e2n + e4n) - (e2o + e4o)
        scale = ref.abs_terms(s, new, i0, j0)
        err = abs(float(rec["dE"]) - d64)
        worst = max(worst, err / scale if scale > 0 else err)
        if d64 != 0.0:
            worst_rel = max(worst_rel, err / abs(d64))
            rels.append(err / abs(d64))
        if g2d is not None:
            # hamiltonian.cu form, computed on its own (g2 over i <= j, hamiltonian.cu:30-38)
            # the interleaved copies must outlive the calls that read them
            flat = [np.ascontiguousarray(np.stack([v.real, v.imag], -1).ravel()) for v in (s, new)]
            hs = [lib().orc_energy_h2_with_diag(len(s), P(g2c), P(f)) for f in flat]
            d_ham = (hs[1] + e4n) - (hs[0] + e4o)
            dd = sum(-g2d[k] * (abs(new[k]) ** 2 - abs(s[k]) ** 2) for k in (i0, j0))   # its diagonal part
            diag_max = max(diag_max, abs(d_ham - d64) / scale if scale > 0 else abs(d_ham - d64))
            ham_err = max(ham_err, abs(float(rec["dE"]) + dd - d_ham) / scale if scale > 0 else 0.0)
        if rec["accepted"]:
            s = new
            e_cur = (e2n, e4n)
        else:
            e_cur = (e2o, e4o)
    if report is not None:
        report.update(n=len(trace), worst=worst, rel_max=worst_rel,
                      rel_median=float(np.median(rels)) if rels else 0.0,
                      diag_max=diag_max if g2d is not None else None,
                      ham_err_max=ham_err if g2d is not None else None)
    return worst, worst_rel, len(trace)


def cpu_sweep_rate(Ns, seeds, NT: int, nrep: int, beta_sched, sweeps: int = 1, nthreads: int = 0,
                   variant: int = 0):
    """Times the CPU transcription of the reference sweep (reference loop
    structure, FP64, OpenMP over replicas; oracle.c orc_sweep) on one sample
    per entry of Ns.  Returns (seconds per sweep for each sample, threads)."""
    import time
    L = lib()
    threads = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    out = []
    for N, seed in zip(Ns, seeds):
        R = NT * nrep
        c = cfg(N=N, nrep=R, seed=seed, fmc_mode=0)
        ref = DenseInit(c)
        betas = np.repeat(np.asarray(beta_sched, np.float64), nrep)
        acc = np.zeros(R, np.int64)
        prop = np.zeros(R, np.int64)
        seeds_r = np.zeros(R, np.uint64)
        L.orc_replica_seeds(seed, R, P(seeds_r))
        ctr = np.zeros(R, np.uint64)
        a = OrcSweepArgs(variant=variant, N=N, nrep=R, h2_active=ref.info.h2_active, g2=P(ref.g2).value,
                         g4=P(ref.g4).value, mask=P(ref.mask).value, nq=0, q_ijklch=None, q_g=None,
                         spins=P(ref.spins).value, energies=P(ref.energies).value, betas=P(betas).value,
                         accepted=P(acc).value, proposed=P(prop).value, seeds=P(seeds_r).value,
                         move_counter=P(ctr).value, nthreads=threads)
        t0 = time.perf_counter()
        L.orc_sweep(ctypes.byref(a), sweeps)
        out.append((time.perf_counter() - t0) / sweeps)
    return out, threads
