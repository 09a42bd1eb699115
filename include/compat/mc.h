/*
 * compat/mc.h -- the reference's dense sweep interface (giacomotrinca/cuda_pspin
 * include/mc.h:9-56) on top of libpspin.
 *
 * Put this directory before the reference's include directory
 * (-I<this repo>/include/compat -I<reference>/include) and link -lpspin:
 * programs written against mc.h -- the reference's drivers and tests --
 * then compile unchanged and run on the B200 engine.  config.h (SimConfig,
 * default_config) stays the reference's; pspin_config has its layout.
 *
 * MCState keeps the fields callers read:
 *   d_accepted, d_proposed, d_energies, d_betas  device pointers into the
 *        engine's own arrays (pspin_device_arrays), so the drivers'
 *        cudaMemset of the counters (parallel_tempering.cu:396-397) works
 *        as written;
 *   d_g2  an FP64 complex copy of the 2-body couplings [N*N] made at init;
 *   h_omega, n_pairs_active, n_quart_active, h2_active, N, nrep.
 * d_g4, d_g4_mask, d_spins and d_rng are NULL: the engine keeps FP32
 * amplitudes and its own coupling layout.  Read couplings and spins with
 * pspin_get_couplings / mc_get_spins instead.
 *
 * Every call is synchronous, as in the reference (mc.cu:799).  Each sweep
 * call first waits for the device (cudaDeviceSynchronize), so writes the
 * caller made through the device pointers on other streams -- the legacy
 * default stream included -- are complete before the engine's stream reads
 * them.  Errors print pspin_last_error() and exit(1), the reference's
 * policy (mc.cu:12-20).
 */
#ifndef MC_H
#define MC_H

#include "config.h"
#include "../pspin.h"

#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <vector>

struct MCState {
    cuDoubleComplex* d_g2;       /* FP64 copy of the 2-body couplings [N*N] */
    cuDoubleComplex* d_g4;       /* NULL (engine layout) */
    uint8_t* d_g4_mask;          /* NULL */
    cuDoubleComplex* d_spins;    /* NULL (FP32 on the engine; mc_get_spins) */
    void* d_rng;                 /* NULL (counter-based streams) */
    double* d_energies;          /* engine's running energies [nrep] */
    long long* d_accepted;       /* engine's counters [nrep] */
    long long* d_proposed;
    double* d_betas;             /* engine's betas [nrep] */
    double* h_omega;             /* host [N], NULL if fully connected */
    long long n_pairs_active;
    long long n_quart_active;
    int h2_active;
    int N;
    int nrep;
    pspin_state* handle;
};

static inline void pspin_compat_check(int rc) {
    if (rc != PSPIN_OK) {
        fprintf(stderr, "pspin: %s\n", pspin_last_error());
        exit(1);
    }
}

static inline void pspin_compat_cuda(cudaError_t e) {
    if (e != cudaSuccess) {
        fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
        exit(1);
    }
}

/* omega (if FMC), counts and the FP64 g2 copy, shared by both shims */
static inline void pspin_compat_fill(pspin_state* h, const SimConfig& cfg, double** h_omega, long long* npa,
                                     long long* nqa, int* h2, cuDoubleComplex** d_g2) {
    pspin_info info;
    pspin_compat_check(pspin_get_info(h, 0, &info));
    *npa = info.n_pairs_active;
    *nqa = info.n_quart_active;
    *h2 = info.h2_active;
    *h_omega = NULL;
    if (cfg.fmc_mode > 0) {
        *h_omega = (double*)malloc(sizeof(double) * (size_t)cfg.N);
        pspin_compat_check(pspin_get_omega(h, 0, *h_omega));
    }
    std::vector<double> g2((size_t)cfg.N * cfg.N * 2);
    pspin_compat_check(pspin_get_couplings(h, 0, g2.data(), NULL, NULL));
    pspin_compat_cuda(cudaMalloc((void**)d_g2, g2.size() * sizeof(double)));
    pspin_compat_cuda(cudaMemcpy(*d_g2, g2.data(), g2.size() * sizeof(double), cudaMemcpyHostToDevice));
}

static inline MCState mc_init(const SimConfig& cfg) {
    MCState s;
    s.handle = NULL;
    pspin_compat_check(pspin_create(reinterpret_cast<const pspin_config*>(&cfg), PSPIN_DENSE, NULL, &s.handle));
    s.N = cfg.N;
    s.nrep = cfg.nrep;
    s.d_g4 = NULL;
    s.d_g4_mask = NULL;
    s.d_spins = NULL;
    s.d_rng = NULL;
    int64_t *acc = NULL, *prop = NULL;
    pspin_compat_check(pspin_device_arrays(s.handle, &acc, &prop, &s.d_energies, &s.d_betas));
    s.d_accepted = reinterpret_cast<long long*>(acc);
    s.d_proposed = reinterpret_cast<long long*>(prop);
    pspin_compat_fill(s.handle, cfg, &s.h_omega, &s.n_pairs_active, &s.n_quart_active, &s.h2_active, &s.d_g2);
    return s;
}

static inline void mc_free(MCState& s) {
    if (s.handle) pspin_destroy(s.handle);
    s.handle = NULL;
    if (s.d_g2) cudaFree(s.d_g2);
    s.d_g2 = NULL;
    free(s.h_omega);
    s.h_omega = NULL;
}

/* mc.cu:746-766: every replica at beta = 1/cfg.T, one sweep */
static inline void mc_sweep(MCState& s, const SimConfig& cfg) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_fill_betas(s.handle, 1.0 / cfg.T));
    pspin_compat_check(pspin_sweep(s.handle, 1));
}

/* mc.cu:784-800: one sweep at the betas set by mc_set_betas */
static inline void mc_sweep_pt(MCState& s) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_sweep(s.handle, 1));
}

static inline void mc_set_betas(MCState& s, const double* h_betas) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_set_betas(s.handle, h_betas));
}

static inline void mc_get_results(const MCState& s, double* E, long long* acc, long long* prop) {
    pspin_compat_cuda(cudaDeviceSynchronize());
    pspin_compat_check(pspin_get_results(s.handle, E, reinterpret_cast<int64_t*>(acc),
                                         reinterpret_cast<int64_t*>(prop)));
}

/* [nrep][N] complex FP64, physical replica order (mc.cu:774-778) */
static inline void mc_get_spins(const MCState& s, cuDoubleComplex* out) {
    pspin_compat_check(pspin_get_spins(s.handle, reinterpret_cast<double*>(out)));
}

static inline void mc_compute_split_energies(const MCState& s, double* e2, double* e4) {
    pspin_compat_check(pspin_split_energies(s.handle, e2, e4));
}

#endif /* MC_H */
