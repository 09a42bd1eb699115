/*
 * compat/mc_sparse.h -- the reference's sparse sweep interface
 * (giacomotrinca/cuda_pspin include/mc_sparse.h:9-61) on top of libpspin.
 *
 * Same use and rules as compat/mc.h.  MCStateSparse keeps the fields the
 * reference's sparse driver and tests read: d_quartets, a device array of
 * the selected quartets in the reference's SparseQuartet layout (48 bytes,
 * coupling at byte 32, mc_sparse.h:9-13) made at init from
 * pspin_get_sparse_quartets, n_quartets, d_g2, and the engine's counters,
 * energies and betas as device pointers.  d_spins and d_rng are NULL.
 */
#ifndef MC_SPARSE_H
#define MC_SPARSE_H

#include "mc.h"

/* one selected (quartet, channel): the reference's layout, so device copies
 * of this array read the same on both sides */
struct SparseQuartet {
    int i, j, k, l;        /* sorted, i < j < k < l */
    int ch;                /* channel 0, 1, 2 */
    cuDoubleComplex g;     /* rescaled coupling (real) */
};
static_assert(sizeof(SparseQuartet) == 48, "SparseQuartet layout");

struct MCStateSparse {
    cuDoubleComplex* d_g2;
    SparseQuartet* d_quartets;
    int n_quartets;
    cuDoubleComplex* d_spins;    /* NULL (FP32 on the engine; mc_sparse_get_spins) */
    void* d_rng;                 /* NULL */
    double* d_energies;
    long long* d_accepted;
    long long* d_proposed;
    double* d_betas;
    double* h_omega;
    long long n_pairs_active;
    long long n_quart_active;
    int h2_active;
    int N;
    int nrep;
    pspin_state* handle;
};

static inline MCStateSparse mc_sparse_init(const SimConfig& cfg) {
    MCStateSparse s;
    s.handle = NULL;
    pspin_compat_check(pspin_create(reinterpret_cast<const pspin_config*>(&cfg), PSPIN_SPARSE, NULL, &s.handle));
    s.N = cfg.N;
    s.nrep = cfg.nrep;
    s.d_spins = NULL;
    s.d_rng = NULL;
    int64_t *acc = NULL, *prop = NULL;
    pspin_compat_check(pspin_device_arrays(s.handle, &acc, &prop, &s.d_energies, &s.d_betas));
    s.d_accepted = reinterpret_cast<long long*>(acc);
    s.d_proposed = reinterpret_cast<long long*>(prop);
    pspin_compat_fill(s.handle, cfg, &s.h_omega, &s.n_pairs_active, &s.n_quart_active, &s.h2_active, &s.d_g2);
    pspin_info info;
    pspin_compat_check(pspin_get_info(s.handle, 0, &info));
    s.n_quartets = info.n_quartets;
    std::vector<int32_t> q((size_t)s.n_quartets * 5);
    std::vector<double> g((size_t)s.n_quartets);
    pspin_compat_check(pspin_get_sparse_quartets(s.handle, 0, q.data(), g.data()));
    std::vector<SparseQuartet> h((size_t)s.n_quartets);
    for (int t = 0; t < s.n_quartets; t++) {
        h[t].i = q[5 * t];
        h[t].j = q[5 * t + 1];
        h[t].k = q[5 * t + 2];
        h[t].l = q[5 * t + 3];
        h[t].ch = q[5 * t + 4];
        h[t].g = make_cuDoubleComplex(g[t], 0.0);
    }
    s.d_quartets = NULL;
    if (s.n_quartets > 0) {
        pspin_compat_cuda(cudaMalloc((void**)&s.d_quartets, h.size() * sizeof(SparseQuartet)));
        pspin_compat_cuda(cudaMemcpy(s.d_quartets, h.data(), h.size() * sizeof(SparseQuartet),
                                     cudaMemcpyHostToDevice));
    }
    return s;
}

static inline void mc_sparse_free(MCStateSparse& s) {
    if (s.handle) pspin_destroy(s.handle);
    s.handle = NULL;
    if (s.d_g2) cudaFree(s.d_g2);
    if (s.d_quartets) cudaFree(s.d_quartets);
    s.d_g2 = NULL;
    s.d_quartets = NULL;
    free(s.h_omega);
    s.h_omega = NULL;
}

static inline void mc_sparse_sweep_pt(MCStateSparse& s) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_sweep(s.handle, 1));
}

static inline void mc_sparse_set_betas(MCStateSparse& s, const double* h_betas) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_set_betas(s.handle, h_betas));
}

static inline void mc_sparse_get_results(const MCStateSparse& s, double* E, long long* acc, long long* prop) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_get_results(s.handle, E, reinterpret_cast<int64_t*>(acc),
                                         reinterpret_cast<int64_t*>(prop)));
}

static inline void mc_sparse_get_spins(const MCStateSparse& s, cuDoubleComplex* out) {
    pspin_compat_check(pspin_get_spins(s.handle, reinterpret_cast<double*>(out)));
}

static inline void mc_sparse_compute_split_energies(const MCStateSparse& s, double* e2, double* e4) {
    pspin_compat_check(pspin_split_energies(s.handle, e2, e4));
}

#endif /* MC_SPARSE_H */
