/*
 * oracle.h -- CPU FP64 restatement of the cuda_pspin hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libpspin.so, the
 * drivers, the Python package) links or calls this code.  It is used by
 * tests/, by __graft_entry__.smoke() as the checker, and by bench.py's
 * cpu_baseline / --impl reference legs as the timed CPU transcription.
 *
 * Every function cites the reference file:line it restates.  The
 * reference is giacomotrinca/cuda_pspin (CUDA C++, FP64).
 *
 * Third-party arithmetic: the reference draws its Gaussian disorder and
 * initial spins from cuRAND's host API (Philox4_32_10,
 * curandGenerateNormalDouble; disorder.cu:61-68, 98-106; spins.cu:75-82).
 * The oracle does not re-derive cuRAND: orc_curand_normals() calls the
 * library's own host generator (curandCreateGeneratorHost), CUDA 12.9's
 * libcurand 10.3.10.  Whether the host generator and the device generator
 * give identical doubles is checked on the GPU by the test suite.
 */
#ifndef PSPIN_ORACLE_H
#define PSPIN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- integer helpers ------------------------------------------------ */
uint64_t orc_splitmix64(uint64_t* state);                          /* mc.cu:42-47 */
void     orc_replica_seeds(uint64_t seed, int nrep, uint64_t* out); /* mc.cu:419-423 */
int64_t  orc_n_quartets(int N);                                     /* disorder.h:32-34 */
int64_t  orc_n_pairs(int N);                                        /* disorder.h:42-44 */
int64_t  orc_encode_quartet(int i, int j, int k, int l);            /* test_quartet_index.cu:28-33 */
void     orc_decode_quartet(int64_t q, int* i, int* j, int* k, int* l); /* mc_sparse.cu:320-335 */
/* 3-type enumeration of the quartets touching (i0,j0) (mc.cu:183-243).
 * Writes n_h4 sorted quartets as 4 ints each; returns n_h4. */
int64_t  orc_three_type(int N, int i0, int j0, int32_t* out_ijkl);

/* ---- configuration ---------------------------------------------------- */
double   orc_auto_gamma(int fmc_mode, int N, double gamma);        /* config.cu:61-67 */
void     orc_temperature_schedule(int NT, double Tmin, double Tmax, int log_temp,
                                  double* T, double* beta);         /* parallel_tempering.cu:93-109 */

/* ---- frequencies and FMC --------------------------------------------- */
void     orc_omega(int N, int fmc_mode, uint64_t seed, double* omega); /* mc.cu:449-460 */
void     orc_fmc_g2(double* g2, int N, const double* omega, double gamma); /* disorder.cu:130-143 */
int64_t  orc_count_pairs_active(const double* g2, int N);          /* mc.cu:469-477 */
void     orc_fmc_g4_mask(uint8_t* mask, int N, const double* omega, double gamma); /* disorder.cu:153-183 */
uint8_t  orc_fmc_channel(int i, int j, int k, int l, const double* omega, double gamma); /* disorder.cu:174-180 */
int64_t  orc_count_active_g4(const uint8_t* mask, int64_t nq);     /* disorder.cu:234-243 */
/* Survivor count by channel for a large N without storing the mask
 * (nested loops in q order).  counts[3]; returns the total. */
int64_t  orc_count_survivors(int N, const double* omega, double gamma, int64_t* counts);

/* ---- cuRAND host generator (library call, not a restatement) -------- */
/* Returns 0 on success.  count must be even. */
int      orc_curand_normals(uint64_t seed, int64_t count, double* out);

/* ---- disorder assembly given raw unit normals ------------------------- */
/* normals for g2: 2*N*N doubles; for g4: 2*C4 doubles (even count). */
void     orc_build_g2(const double* normals, int N, double* g2);   /* disorder.cu:57-80 */
void     orc_build_g4(const double* normals, int64_t nq, double* g4); /* disorder.cu:93-113 */
void     orc_scale(double* c, int64_t n, double sigma);            /* disorder.cu:28-35 */
void     orc_shift_mean(double* c, int64_t n, double mean);        /* disorder.cu:200-216 */

typedef struct orc_config {            /* mirrors SimConfig, config.h:9-25 */
    int save_freq, verbose, N, nrep;
    double T, J, J0, alpha, alpha0;
    int mc_iterations;
    uint64_t seed;
    int label, dev, fmc_mode;
    double gamma;
} orc_config;

typedef struct orc_disorder_info {
    int64_t n_pairs_active;
    int64_t n_quart_active;
    int     h2_active;
    int     n_sparse;                  /* sparse variant: selected quartets */
} orc_disorder_info;

/* mc_init (mc.cu:411-562) for the dense variant.
 * Outputs (caller allocates): g2 [N*N*2], g4 [C4*2], mask [C4],
 * omega [N] (may be NULL when fmc==0), spins [nrep*N*2],
 * energies [nrep] (chain form).  init_exact != 0 replaces the reference's
 * truncated tree reduction (spins.cu:27-69) by a full sum. */
int      orc_init_dense(const orc_config* cfg, int init_exact,
                        double* g2, double* g4, uint8_t* mask, double* omega,
                        double* spins, double* energies, orc_disorder_info* info);

/* mc_sparse_init (mc_sparse.cu:390-604).  q_ijklch [N*5], q_g [N].
 * Needs C(N,4) normals: only for small N (the GPU test at N=512 uses
 * orc_sparse_select below). */
int      orc_init_sparse(const orc_config* cfg, int init_exact,
                         double* g2, int32_t* q_ijklch, double* q_g, double* omega,
                         double* spins, double* energies, orc_disorder_info* info);

/* Sparse selection only (mc_sparse.cu:489-537 without the coupling values):
 * survivors in ascending q*3+ch order, partial Fisher-Yates with
 * splitmix64(seed+4000).  Returns selected encodings q*3+ch in out_enc
 * (n_select entries) and the survivor count in *n_nonzero.  Works for
 * N=512 (streams the survivors, 8 bytes each). */
int      orc_sparse_select(int N, const double* omega, double gamma, int fmc_mode,
                           uint64_t seed, int n_select, int64_t* out_enc, int64_t* n_nonzero);
void     orc_partial_shuffle(int64_t* arr, int64_t count, int n_select, uint64_t seed); /* mc_sparse.cu:340-349 */

/* ---- spins -------------------------------------------------------------- */
void     orc_normalize_sphere(double* spins, int N, int exact);    /* spins.cu:27-69 (F8 tree) */
void     orc_normalize_cube(double* spins, int N, int exact);      /* spins_sparse.cu:28-61 */

/* ---- energies (chain form: g2 i<j, no diagonal) ------------------------ */
void     orc_energy_dense(int N, const double* g2, const double* g4, const uint8_t* mask,
                          int h2_active, const double* spins, double* e2, double* e4); /* mc.cu:323-405, 567-656 */
void     orc_energy_sparse(int N, const double* g2, int nq, const int32_t* q_ijklch,
                           const double* q_g, int h2_active, const double* spins,
                           double* e2, double* e4);                /* mc_sparse.cu:258-315 */
/* hamiltonian.cu form: H2 over i<=j including the diagonal (hamiltonian.cu:23-58) */
double   orc_energy_h2_with_diag(int N, const double* g2, const double* spins);
/* Sum of |terms| over the quartets/pairs touching (i0,j0), old and new
 * spins: the scale the per-move dE tolerance is relative to. */
double   orc_dense_abs_terms(int N, const double* g2, const double* g4, const uint8_t* mask,
                             int h2_active, const double* spins_old, const double* spins_new,
                             int i0, int j0);
double   orc_sparse_abs_terms(int N, const double* g2, int nq, const int32_t* q_ijklch,
                              const double* q_g, int h2_active, const double* spins_old,
                              const double* spins_new, int i0, int j0);

/* ---- proposals (given uniforms) ---------------------------------------- */
void     orc_propose_sphere(const double* ai, const double* aj, double u_alpha,
                            double u_phi1, double u_phi2, double* ai_new, double* aj_new); /* spins.h:17-52 */
void     orc_propose_cube(const double* ai, const double* aj, double u, double u_phi1,
                          double u_phi2, double* ai_new, double* aj_new); /* spins_sparse.h:26-56 */

/* ---- random streams ---------------------------------------------------- */
/* Philox4x32-10, Salmon, Moraes, Dror & Shaw, SC'11 (Random123). */
void     orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* POSIX drand48 LCG: X <- 0x5DEECE66D*X + 0xB mod 2^48. */
uint64_t orc_srand48_state(long seedval);
double   orc_drand48(uint64_t* state);

/* ---- replica exchange (parallel_tempering.cu:316-352) ---------------- */
void     orc_exchange(int NT, int nrep_per_temp, const double* beta_sched,
                      const double* energies, int32_t* perm, uint64_t* drand_state,
                      int64_t* ex_acc, int64_t* ex_prop, double* betas_out);

/* ---- CPU sweep (reference loop structure, FP64, OpenMP over replicas) --
 * The timed CPU baseline and the statistical checker.  RNG: Philox4x32-10
 * keyed by the replica seed (the reference uses cuRAND's device Philox, whose
 * output mapping is not restated here).  Per move: pair pick, proposal,
 * H2+H4 dE by the reference's 3-type enumeration (mc.cu:126-306).
 * variant 0 = dense sphere (g4 dense + mask), 1 = sparse cube (quartet list).
 * move_counter: per-replica 64-bit counters (advanced in place). */
typedef struct orc_sweep_args {
    int variant, N, nrep, h2_active;
    const double* g2; const double* g4; const uint8_t* mask;          /* dense */
    int nq; const int32_t* q_ijklch; const double* q_g;               /* sparse */
    double* spins; double* energies; const double* betas;
    int64_t* accepted; int64_t* proposed;
    const uint64_t* seeds; uint64_t* move_counter;
    int nthreads;
} orc_sweep_args;
void     orc_sweep(orc_sweep_args* a, int nsweeps);

#ifdef __cplusplus
}
#endif
#endif
