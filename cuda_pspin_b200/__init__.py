"""B200 Monte Carlo engine for the complex 2+4 p-spin glass.

Python face of ``libpspin.so`` (the C ABI in ``include/pspin.h``).  The
function names mirror the reference's sweep interface (mc.h:33-56,
mc_sparse.h:42-61): ``mc_init``, ``mc_sweep``, ``mc_sweep_pt``,
``mc_set_betas``, ``mc_get_results``, ``mc_get_spins``,
``mc_compute_split_energies``, ``mc_free`` and the ``mc_sparse_*`` twins.
Where the reference calls ``exit(1)`` these raise :class:`PspinError`.

The library is built in-tree (``python -m cuda_pspin_b200.build``).  There is
no CPU fallback: importing works without a GPU, but every call that needs the
device raises if the CUDA library or the GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpspin.so")
BIN_DIR = os.path.join(_HERE, "bin")

PSPIN_DENSE = 0
PSPIN_SPARSE = 1
FIELDS_FP64 = 0
FIELDS_TC_BF16X3 = 1
RESYNC_FP64 = 0
RESYNC_TC = 1
PROPOSAL_PLAIN = 0
PROPOSAL_PLAIN_FIELDS = 1
PROPOSAL_LEARNED = 2
MLP_PARAMS = 6426
RECORD_FLOATS = 11
PSPIN_OK = 0
PSPIN_ERR_ARG = 1
PSPIN_ERR_TIMEOUT = 8
_STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_CURAND", 4: "ERR_ALLOC", 5: "ERR_STATE",
           6: "ERR_NUMERIC", 7: "ERR_UNSUPPORTED", 8: "ERR_TIMEOUT"}


class PspinError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


class SimConfig(ctypes.Structure):
    """Same layout as the reference's SimConfig (config.h:9-25)."""
    _fields_ = [("save_freq", ctypes.c_int), ("verbose", ctypes.c_int), ("N", ctypes.c_int),
                ("nrep", ctypes.c_int), ("T", ctypes.c_double), ("J", ctypes.c_double),
                ("J0", ctypes.c_double), ("alpha", ctypes.c_double), ("alpha0", ctypes.c_double),
                ("mc_iterations", ctypes.c_int), ("seed", ctypes.c_uint64), ("label", ctypes.c_int),
                ("dev", ctypes.c_int), ("fmc_mode", ctypes.c_int), ("gamma", ctypes.c_double)]

    def __repr__(self) -> str:
        return "SimConfig(" + ", ".join(f"{n}={getattr(self, n)!r}" for n, _ in self._fields_) + ")"


class Options(ctypes.Structure):
    _fields_ = [("init_exact", ctypes.c_int), ("resync_every", ctypes.c_int),
                ("warps_per_unit", ctypes.c_int), ("trace_sample", ctypes.c_int),
                ("trace_replica", ctypes.c_int), ("trace_capacity", ctypes.c_int),
                ("quiet", ctypes.c_int), ("generic_lists", ctypes.c_int), ("graph_steps", ctypes.c_int),
                ("resync_method", ctypes.c_int), ("cluster_size", ctypes.c_int),
                ("wait_limit_clocks", ctypes.c_int), ("test_stall_move", ctypes.c_int),
                ("disorder_stream", ctypes.c_int), ("replicas_per_lane", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("nrep", ctypes.c_int), ("h2_active", ctypes.c_int),
                ("n_quartets", ctypes.c_int), ("n_pairs_active", ctypes.c_int64),
                ("n_quart_active", ctypes.c_int64), ("site_entries", ctypes.c_int64)]


MOVE_RECORD = np.dtype([("i0", np.int32), ("j0", np.int32), ("ai_old", np.float32, 2),
                        ("aj_old", np.float32, 2), ("ai_new", np.float32, 2), ("aj_new", np.float32, 2),
                        ("dE", np.float32), ("accepted", np.int32), ("log_q_ratio", np.float32),
                        ("log_u", np.float32)])

_lib = None


def load_library() -> ctypes.CDLL:
    """Load libpspin.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cuda_pspin_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sig = {
        "pspin_default_config": (None, [P(SimConfig)]),
        "pspin_parse_args": (ctypes.c_int, [ctypes.c_int, P(ctypes.c_char_p), P(SimConfig)]),
        "pspin_create": (ctypes.c_int, [P(SimConfig), ctypes.c_int, P(Options), P(vp)]),
        "pspin_create_batch": (ctypes.c_int, [P(SimConfig), ctypes.c_int, ctypes.c_int, P(Options), P(vp)]),
        "pspin_destroy": (ctypes.c_int, [vp]),
        "pspin_set_betas": (ctypes.c_int, [vp, vp]),
        "pspin_fill_betas": (ctypes.c_int, [vp, ctypes.c_double]),
        "pspin_sweep": (ctypes.c_int, [vp, ctypes.c_int]),
        "pspin_get_results": (ctypes.c_int, [vp, vp, vp, vp]),
        "pspin_reset_counters": (ctypes.c_int, [vp]),
        "pspin_get_spins": (ctypes.c_int, [vp, vp]),
        "pspin_set_spins": (ctypes.c_int, [vp, vp]),
        "pspin_split_energies": (ctypes.c_int, [vp, vp, vp]),
        "pspin_resync": (ctypes.c_int, [vp]),
        "pspin_total_replicas": (ctypes.c_int, [vp]),
        "pspin_num_samples": (ctypes.c_int, [vp]),
        "pspin_get_info": (ctypes.c_int, [vp, ctypes.c_int, P(Info)]),
        "pspin_get_omega": (ctypes.c_int, [vp, ctypes.c_int, vp]),
        "pspin_get_couplings": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp]),
        "pspin_get_sparse_quartets": (ctypes.c_int, [vp, ctypes.c_int, vp, vp]),
        "pspin_pt_init": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]),
        "pspin_pt_run": (ctypes.c_int, [vp, ctypes.c_int]),
        "pspin_pt_get": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp]),
        "pspin_pt_sweeps_done": (ctypes.c_int, [vp, vp]),
        "pspin_trace_get": (ctypes.c_int, [vp, vp, ctypes.c_int, vp]),
        "pspin_fmc_mask": (ctypes.c_int, [ctypes.c_int, vp, ctypes.c_double, vp, vp]),
        "pspin_quartet_roundtrip": (ctypes.c_int, [ctypes.c_int, vp]),
        "pspin_fmc_survivors_static": (ctypes.c_int, [ctypes.c_int, vp, ctypes.c_double, vp, vp]),
        "pspin_local_fields": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, vp]),
        "pspin_sweep_work": (ctypes.c_int, [vp, vp, vp]),
        "pspin_device_arrays": (ctypes.c_int, [vp, vp, vp, vp, vp]),
        "pspin_deeper_counts": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_double, vp, ctypes.c_int,
                                               vp, vp, vp, vp, vp]),
        "pspin_multi_overlap": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp,
                                               ctypes.c_int, vp]),
        "pspin_std_shuffle": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, vp]),
        "pspin_reservoir_sample": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, vp, ctypes.c_int,
                                                  ctypes.c_uint32, vp, vp]),
        "pspin_fy_downsample": (ctypes.c_int, [ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_uint32,
                                               vp, vp]),
        "pspin_tau_e": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, vp]),
        "pspin_shard_samples": (ctypes.c_int, [ctypes.c_int, vp, vp, ctypes.c_int, vp]),
        "pspin_cube_samples": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, vp]),
        "pspin_cube_walk": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, vp,
                                           ctypes.c_int, vp]),
        "pspin_set_proposal": (ctypes.c_int, [vp, ctypes.c_int]),
        "pspin_observe_init": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
        "pspin_autotune": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp]),
        "pspin_autotune_lanes": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp, vp]),
        "pspin_resync_drift": (ctypes.c_int, [vp, vp]),
        "pspin_checkpoint_save": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "pspin_pt_shape": (ctypes.c_int, [vp, vp, vp, vp]),
        "pspin_overlap_counts": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double, vp]),
        "pspin_ifo_counts": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double, vp, vp, vp, vp]),
        "pspin_exchange_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp,
                                               vp]),
        "pspin_checkpoint_load": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "pspin_observe_get": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int]),
        "pspin_learn_init": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_float]),
        "pspin_learn_params": (ctypes.c_int, [vp, vp, vp]),
        "pspin_learn_train": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, vp]),
        "pspin_learn_records": (ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
        "pspin_learn_loss_grad": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, vp]),
        "pspin_stream": (vp, [vp]),
        "pspin_set_profiling": (ctypes.c_int, [vp, ctypes.c_int]),
        "pspin_get_profile": (ctypes.c_int, [vp, vp, vp, vp]),
        "pspin_fp32_peak": (ctypes.c_int, [vp]),
        "pspin_last_error": (ctypes.c_char_p, []),
        "pspin_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise PspinError(rc, load_library().pspin_last_error().decode())


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def default_config(**kw) -> SimConfig:
    """config.h:28-46, with keyword overrides."""
    c = SimConfig()
    load_library().pspin_default_config(ctypes.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def parse_args(argv: list[str]) -> SimConfig:
    """config.cu:6-70 (raises PspinError where the reference exits)."""
    c = SimConfig()
    arr = (ctypes.c_char_p * len(argv))(*[a.encode() for a in argv])
    _check(load_library().pspin_parse_args(len(argv), arr, ctypes.byref(c)))
    return c


def make_options(init_exact: bool = False, resync_every: int = 0, warps_per_unit: int = 0,
                 trace: tuple[int, int, int] | None = None, quiet: bool = True,
                 generic_lists: bool = False, graph_steps: int = 0, resync_method: int = 0,
                 cluster_size: int = 0, wait_limit_clocks: int = 0, test_stall_move: int = 0,
                 disorder_stream: bool = False, replicas_per_lane: int = 0) -> Options:
    o = Options()
    o.disorder_stream = int(disorder_stream)
    o.replicas_per_lane = int(replicas_per_lane)
    o.cluster_size = int(cluster_size)
    o.wait_limit_clocks = int(wait_limit_clocks)
    o.test_stall_move = int(test_stall_move)
    o.resync_method = int(resync_method)
    o.generic_lists = int(generic_lists)
    o.graph_steps = int(graph_steps)
    o.init_exact = int(init_exact)
    o.resync_every = resync_every
    o.warps_per_unit = warps_per_unit
    if trace is None:
        o.trace_sample, o.trace_replica, o.trace_capacity = 0, -1, 0
    else:
        o.trace_sample, o.trace_replica, o.trace_capacity = trace
    o.quiet = int(quiet)
    return o


class Engine:
    """A batch of disorder samples resident on the GPU (one handle)."""

    def __init__(self, cfgs, variant: int = PSPIN_DENSE, options: Options | None = None):
        lib = load_library()
        if isinstance(cfgs, SimConfig):
            cfgs = [cfgs]
        arr = (SimConfig * len(cfgs))(*cfgs)
        h = ctypes.c_void_p()
        opt = options if options is not None else make_options()
        _check(lib.pspin_create_batch(arr, len(cfgs), variant, ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self.variant = variant
        self.cfgs = list(cfgs)
        self.n_samples = len(cfgs)
        self.n_replicas = lib.pspin_total_replicas(h)
        self.Ns = [c.N for c in cfgs]
        self.Rs = [c.nrep for c in cfgs]

    # -- lifetime ----------------------------------------------------------
    def free(self) -> None:
        if self._h:
            _check(self._lib.pspin_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    # -- sweep interface -----------------------------------------------------
    def set_betas(self, betas) -> None:
        b = np.ascontiguousarray(betas, dtype=np.float64)
        assert b.shape == (self.n_replicas,)
        _check(self._lib.pspin_set_betas(self._h, _ptr(b)))

    def fill_betas(self, beta: float) -> None:
        _check(self._lib.pspin_fill_betas(self._h, float(beta)))

    def sweep(self, nsweeps: int = 1) -> None:
        _check(self._lib.pspin_sweep(self._h, int(nsweeps)))

    def get_results(self):
        E = np.empty(self.n_replicas, np.float64)
        a = np.empty(self.n_replicas, np.int64)
        p = np.empty(self.n_replicas, np.int64)
        _check(self._lib.pspin_get_results(self._h, _ptr(E), _ptr(a), _ptr(p)))
        return E, a, p

    def reset_counters(self) -> None:
        _check(self._lib.pspin_reset_counters(self._h))

    def get_spins(self) -> list[np.ndarray]:
        """Per sample, complex128 [nrep, N] (physical replica order)."""
        tot = sum(N * R for N, R in zip(self.Ns, self.Rs))
        buf = np.empty(2 * tot, np.float64)
        _check(self._lib.pspin_get_spins(self._h, _ptr(buf)))
        out, off = [], 0
        for N, R in zip(self.Ns, self.Rs):
            v = buf[2 * off:2 * (off + N * R)].reshape(R, N, 2)
            out.append(v[..., 0] + 1j * v[..., 1])
            off += N * R
        return out

    def set_spins(self, spins: list[np.ndarray]) -> None:
        parts = []
        for s in spins:
            s = np.asarray(s, np.complex128)
            parts.append(np.stack([s.real, s.imag], -1).ravel())
        buf = np.ascontiguousarray(np.concatenate(parts))
        _check(self._lib.pspin_set_spins(self._h, _ptr(buf)))

    def split_energies(self):
        e2 = np.empty(self.n_replicas, np.float64)
        e4 = np.empty(self.n_replicas, np.float64)
        _check(self._lib.pspin_split_energies(self._h, _ptr(e2), _ptr(e4)))
        return e2, e4

    def resync(self) -> None:
        _check(self._lib.pspin_resync(self._h))

    # -- disorder introspection ----------------------------------------------
    def info(self, sample: int = 0) -> Info:
        i = Info()
        _check(self._lib.pspin_get_info(self._h, sample, ctypes.byref(i)))
        return i

    def omega(self, sample: int = 0) -> np.ndarray:
        w = np.empty(self.Ns[sample], np.float64)
        _check(self._lib.pspin_get_omega(self._h, sample, _ptr(w)))
        return w

    def couplings(self, sample: int = 0, dense_g4: bool = True):
        N = self.Ns[sample]
        g2 = np.empty(2 * N * N, np.float64)
        if dense_g4 and self.variant == PSPIN_DENSE:
            nq = N * (N - 1) * (N - 2) * (N - 3) // 24
            g4 = np.empty(2 * nq, np.float64)
            m = np.empty(nq, np.uint8)
            _check(self._lib.pspin_get_couplings(self._h, sample, _ptr(g2), _ptr(g4), _ptr(m)))
            return g2.reshape(N, N, 2)[..., 0], g4[0::2].copy(), m
        _check(self._lib.pspin_get_couplings(self._h, sample, _ptr(g2), None, None))
        return g2.reshape(N, N, 2)[..., 0], None, None

    def sparse_quartets(self, sample: int = 0):
        n = self.info(sample).n_quartets
        q = np.empty(5 * n, np.int32)
        g = np.empty(n, np.float64)
        _check(self._lib.pspin_get_sparse_quartets(self._h, sample, _ptr(q), _ptr(g)))
        return q.reshape(n, 5), g

    # -- parallel tempering ----------------------------------------------------
    def pt_init(self, NT: int, nrep_per_temp: int, beta_sched, pt_freq: int = 1) -> None:
        b = np.ascontiguousarray(beta_sched, dtype=np.float64)
        _check(self._lib.pspin_pt_init(self._h, NT, nrep_per_temp, _ptr(b), pt_freq))
        self.NT, self.nrep_per_temp = NT, nrep_per_temp

    def pt_run(self, nsweeps: int) -> None:
        _check(self._lib.pspin_pt_run(self._h, int(nsweeps)))

    def pt_get(self, sample: int = 0):
        NT, nr = self.NT, self.nrep_per_temp
        perm = np.empty(NT * nr, np.int32)
        acc = np.empty(NT - 1, np.int64)
        prop = np.empty(NT - 1, np.int64)
        _check(self._lib.pspin_pt_get(self._h, sample, _ptr(perm), _ptr(acc), _ptr(prop)))
        return perm, acc, prop

    def checkpoint_save(self, path: str) -> None:
        _check(self._lib.pspin_checkpoint_save(self._h, os.fsencode(path)))

    def checkpoint_load(self, path: str) -> None:
        """Restores a checkpoint written by a handle built from the same configurations."""
        _check(self._lib.pspin_checkpoint_load(self._h, os.fsencode(path)))
        NT, nr, fq = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(self._lib.pspin_pt_shape(self._h, ctypes.byref(NT), ctypes.byref(nr), ctypes.byref(fq)))
        if NT.value >= 2:
            self.NT, self.nrep_per_temp = NT.value, nr.value

    def resync_drift(self) -> np.ndarray:
        """|E_running - E_recomputed| per replica at the last periodic resync."""
        d = np.empty(self.n_replicas, np.float64)
        _check(self._lib.pspin_resync_drift(self._h, _ptr(d)))
        return d

    def autotune(self, sweeps: int = 8):
        """(warps per CTA, CTAs per replica block (0: list-resident one-warp kernel),
        ms per sweep [resident, cluster 1, 2, 4, 8, 16][warps 1, 2, 4, 8])."""
        w, c = ctypes.c_int(0), ctypes.c_int(0)
        ms = np.zeros((6, 4), np.float32)
        _check(self._lib.pspin_autotune(self._h, int(sweeps), ctypes.byref(w), ctypes.byref(c), _ptr(ms)))
        return w.value, c.value, ms

    def autotune_lanes(self, sweeps: int = 8):
        """Plain sweep: (warps, cluster, replicas per lane, ms per sweep
        [replicas per lane 1, 2, 3][resident, cluster 1, 2, 4, 8, 16][warps 1, 2, 4, 8])."""
        w, c, k = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        ms = np.zeros((3, 6, 4), np.float32)
        _check(self._lib.pspin_autotune_lanes(self._h, int(sweeps), ctypes.byref(w), ctypes.byref(c),
                                              ctypes.byref(k), _ptr(ms)))
        return w.value, c.value, k.value, ms

    def observe_init(self, temp_index: int, capacity: int) -> None:
        _check(self._lib.pspin_observe_init(self._h, int(temp_index), int(capacity)))

    def observe_get(self):
        """(E [rows, samples, nrep], q [rows, samples, nrep(nrep-1)/2]) at the observed slot."""
        nr = self.nrep_per_temp
        npairs = nr * (nr - 1) // 2
        n = ctypes.c_int64(0)
        _check(self._lib.pspin_observe_get(self._h, ctypes.byref(n), None, None, 0))
        rows = n.value
        E = np.empty((max(rows, 1), self.n_samples, nr), np.float64)
        q = np.empty((max(rows, 1), self.n_samples, max(npairs, 1)), np.float64)
        _check(self._lib.pspin_observe_get(self._h, ctypes.byref(n), _ptr(E), _ptr(q), rows))
        return E[:rows], q[:rows, :, :npairs]

    # -- all-site local fields ------------------------------------------------------
    def local_fields(self, sample: int = 0, method: int = 0):
        """(h [nrep, N] complex, energy [nrep]); method FIELDS_FP64 or FIELDS_TC_BF16X3."""
        N, R = self.Ns[sample], self.Rs[sample]
        h = np.empty(2 * N * R, np.float64)
        e = np.empty(R, np.float64)
        _check(self._lib.pspin_local_fields(self._h, sample, method, _ptr(h), _ptr(e)))
        v = h.reshape(R, N, 2)
        return v[..., 0] + 1j * v[..., 1], e

    # -- learned proposal -------------------------------------------------------------
    def set_proposal(self, proposal: int) -> None:
        _check(self._lib.pspin_set_proposal(self._h, int(proposal)))

    def learn_init(self, seed: int = 1, capacity: int = 1 << 20, record_prob: float = 1.0) -> None:
        _check(self._lib.pspin_learn_init(self._h, int(seed), int(capacity), float(record_prob)))

    def learn_params(self, set_to=None) -> np.ndarray:
        out = np.empty(MLP_PARAMS, np.float32)
        w = None if set_to is None else np.ascontiguousarray(set_to, np.float32)   # alive across the call
        _check(self._lib.pspin_learn_params(self._h, _ptr(out), None if w is None else _ptr(w)))
        if w is not None:
            out = w.copy()
        return out

    def learn_train(self, steps: int, batch: int = 4096, lr: float = 1e-3) -> float:
        loss = ctypes.c_double(0)
        _check(self._lib.pspin_learn_train(self._h, int(steps), int(batch), float(lr), ctypes.byref(loss)))
        return loss.value

    def learn_records(self, max_records: int = 0):
        n = ctypes.c_int64(0)
        out = np.empty((max(max_records, 1), RECORD_FLOATS), np.float32)
        _check(self._lib.pspin_learn_records(self._h, ctypes.byref(n), _ptr(out), int(max_records)))
        return n.value, out[:min(max_records, n.value)]

    def learn_loss_grad(self, records: np.ndarray):
        r = np.ascontiguousarray(records, np.float32)
        loss = ctypes.c_double(0)
        g = np.empty(MLP_PARAMS, np.float32)
        _check(self._lib.pspin_learn_loss_grad(self._h, _ptr(r), len(r), ctypes.byref(loss), _ptr(g)))
        return loss.value, g

    # -- measurement -------------------------------------------------------------
    def sweep_work(self):
        """(algorithmic, executed) FP32 operations of one sweep of every
        sample and replica (pspin_sweep_work)."""
        a, e = ctypes.c_double(), ctypes.c_double()
        _check(self._lib.pspin_sweep_work(self._h, ctypes.byref(a), ctypes.byref(e)))
        return a.value, e.value

    def stream_ptr(self) -> int:
        return int(self._lib.pspin_stream(self._h) or 0)

    def set_profiling(self, on: bool) -> None:
        _check(self._lib.pspin_set_profiling(self._h, int(on)))

    def get_profile(self):
        ms = ctypes.c_double(0)
        sl = ctypes.c_int64(0)
        kl = ctypes.c_int64(0)
        _check(self._lib.pspin_get_profile(self._h, ctypes.byref(ms), ctypes.byref(sl), ctypes.byref(kl)))
        return ms.value, sl.value, kl.value

    def trace(self, max_records: int = 1 << 20) -> np.ndarray:
        out = np.zeros(max_records, MOVE_RECORD)
        n = ctypes.c_int(0)
        _check(self._lib.pspin_trace_get(self._h, _ptr(out), max_records, ctypes.byref(n)))
        return out[:n.value]


# ---- the reference's function names (mc.h:33-56, mc_sparse.h:42-61) --------
def mc_init(cfg: SimConfig, options: Options | None = None) -> Engine:
    return Engine(cfg, PSPIN_DENSE, options)


def mc_sparse_init(cfg: SimConfig, options: Options | None = None) -> Engine:
    return Engine(cfg, PSPIN_SPARSE, options)


def mc_free(state: Engine) -> None:
    state.free()


mc_sparse_free = mc_free


def mc_sweep(state: Engine, cfg: SimConfig) -> None:
    """mc.cu:746-766: betas <- 1/T, one sweep."""
    state.fill_betas(1.0 / cfg.T)
    state.sweep(1)


def mc_sweep_pt(state: Engine) -> None:
    state.sweep(1)


mc_sparse_sweep_pt = mc_sweep_pt


def mc_set_betas(state: Engine, betas) -> None:
    state.set_betas(betas)


mc_sparse_set_betas = mc_set_betas


def mc_get_results(state: Engine):
    return state.get_results()


mc_sparse_get_results = mc_get_results


def mc_get_spins(state: Engine) -> np.ndarray:
    return state.get_spins()[0]


mc_sparse_get_spins = mc_get_spins


def mc_compute_split_energies(state: Engine):
    return state.split_energies()


mc_sparse_compute_split_energies = mc_compute_split_energies


def exchange_host(beta_sched, energy, rep_off, perm, drand_state, ex_acc, ex_prop, betas=None) -> None:
    """The reference's host-side replica exchange (parallel_tempering.cu:316-352)
    in place on caller arrays: perm int32 [S, NT*nrep], drand_state uint64 [S],
    ex_acc / ex_prop int64 [S, NT-1], energy / betas float64 indexed by
    rep_off[k] + physical replica."""
    S, NTn = perm.shape
    NT = len(beta_sched)
    for a, dt in ((perm, np.int32), (drand_state, np.uint64), (ex_acc, np.int64), (ex_prop, np.int64),
                  (energy, np.float64), (rep_off, np.int64)):
        if a.dtype != dt or not a.flags.c_contiguous:
            raise TypeError("exchange_host: arrays must be C-contiguous with the documented dtypes")
    bs = np.ascontiguousarray(beta_sched, np.float64)
    if betas is not None and (betas.dtype != np.float64 or not betas.flags.c_contiguous):
        raise TypeError("exchange_host: betas must be C-contiguous float64")
    _check(load_library().pspin_exchange_host(S, NT, NTn // NT, _ptr(bs), _ptr(energy), _ptr(rep_off), _ptr(perm),
                                              _ptr(drand_state), _ptr(ex_acc), _ptr(ex_prop),
                                              None if betas is None else _ptr(betas)))


def fmc_mask(N: int, omega, gamma: float):
    """disorder.cu:153-183 on the GPU: (mask[C(N,4)], popcount)."""
    w = np.ascontiguousarray(omega, dtype=np.float64)
    nq = N * (N - 1) * (N - 2) * (N - 3) // 24
    m = np.empty(nq, np.uint8)
    n = ctypes.c_int64(0)
    _check(load_library().pspin_fmc_mask(N, _ptr(w), float(gamma), _ptr(m), ctypes.byref(n)))
    return m, n.value


def shard_samples(Ns, Rs, nshards: int) -> np.ndarray:
    """Shard of every sample (pspin_shard_samples: cost N^4 R, largest first
    to the least-loaded shard); the same on every rank."""
    N = np.ascontiguousarray(Ns, np.int32)
    R = np.ascontiguousarray(np.broadcast_to(np.asarray(Rs, np.int32), N.shape), np.int32)
    out = np.zeros(len(N), np.int32)
    _check(load_library().pspin_shard_samples(len(N), _ptr(N), _ptr(R), int(nshards), _ptr(out)))
    return out


def fp32_peak_tflops() -> float:
    t = ctypes.c_double(0)
    _check(load_library().pspin_fp32_peak(ctypes.byref(t)))
    return t.value


def quartet_roundtrip(N: int) -> int:
    n = ctypes.c_int64(0)
    _check(load_library().pspin_quartet_roundtrip(N, ctypes.byref(n)))
    return n.value


def temperature_schedule(NT: int, Tmin: float, Tmax: float, log_temp: bool):
    """parallel_tempering.cu:93-109 (index 0 hottest)."""
    t = np.arange(NT, dtype=np.float64)
    if log_temp:
        A = (Tmin / Tmax) ** (1.0 / (NT - 1)) if NT > 1 else 1.0
        T = np.array([Tmax * A ** k for k in range(NT)])
    else:
        dT = (Tmax - Tmin) / (NT - 1) if NT > 1 else 0.0
        T = Tmax - t * dT
    return T, 1.0 / T


@dataclass
class Workload:
    """Pair-moves of a PT run: replicas x N/2 x sweeps, summed over samples."""
    Ns: list
    Rs: list

    def moves_per_sweep(self) -> int:
        return int(sum(R * (N // 2) for N, R in zip(self.Ns, self.Rs)))
