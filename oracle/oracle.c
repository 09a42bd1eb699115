/*
 * oracle.c -- CPU FP64 restatement of the cuda_pspin hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each function cites the
 * reference file:line whose arithmetic it restates; where the order of
 * floating-point operations decides bit-exactness (FMC tests, the spin
 * normalisation tree, rescale) the reference's order is kept.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <curand.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* integer helpers                                                      */
/* ------------------------------------------------------------------ */

/* mc.cu:42-47 (same constants in mc_sparse.cu:38-43) */
uint64_t orc_splitmix64(uint64_t* state) {
    uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* mc.cu:419-423: one splitmix64 draw per replica from the master seed */
void orc_replica_seeds(uint64_t seed, int nrep, uint64_t* out) {
    uint64_t master = seed;
    for (int r = 0; r < nrep; r++) out[r] = orc_splitmix64(&master);
}

/* disorder.h:32-34 */
int64_t orc_n_quartets(int N) {
    return (int64_t)N * (N - 1) * (N - 2) * (N - 3) / 24;
}

/* disorder.h:42-44 (includes the diagonal) */
int64_t orc_n_pairs(int N) { return (int64_t)N * (N + 1) / 2; }

/* test_quartet_index.cu:28-33, mc.cu:241-243 */
int64_t orc_encode_quartet(int ii, int jj, int kk, int ll) {
    return (int64_t)ll * (ll - 1) * (ll - 2) * (ll - 3) / 24
         + (int64_t)kk * (kk - 1) * (kk - 2) / 6
         + (int64_t)jj * (jj - 1) / 2 + ii;
}

/* mc_sparse.cu:320-335 (linear scans, identical in disorder.cu:158-171) */
void orc_decode_quartet(int64_t q, int* ii, int* jj, int* kk, int* ll) {
    int l = 3;
    while ((int64_t)l * (l - 1) * (l - 2) * (l - 3) / 24 <= q) l++;
    l--;
    int64_t rem = q - (int64_t)l * (l - 1) * (l - 2) * (l - 3) / 24;
    int k = 2;
    while ((int64_t)k * (k - 1) * (k - 2) / 6 <= rem) k++;
    k--;
    rem -= (int64_t)k * (k - 1) * (k - 2) / 6;
    int j = 1;
    while ((int64_t)j * (j - 1) / 2 <= rem) j++;
    j--;
    rem -= (int64_t)j * (j - 1) / 2;
    *ii = (int)rem; *jj = j; *kk = k; *ll = l;
}

static void sort4(int* idx) {   /* mc.cu:234-238 (5-comparator network) */
    int t;
    if (idx[0] > idx[1]) { t = idx[0]; idx[0] = idx[1]; idx[1] = t; }
    if (idx[2] > idx[3]) { t = idx[2]; idx[2] = idx[3]; idx[3] = t; }
    if (idx[0] > idx[2]) { t = idx[0]; idx[0] = idx[2]; idx[2] = t; }
    if (idx[1] > idx[3]) { t = idx[1]; idx[1] = idx[3]; idx[3] = t; }
    if (idx[1] > idx[2]) { t = idx[1]; idx[1] = idx[2]; idx[2] = t; }
}

/* combinatorial decode of the type-1/2 index (mc.cu:189-201) */
static void decode_triple(int64_t tt, int* aa, int* bb, int* cc_out) {
    int cc = (int)cbrt(6.0 * (double)tt);
    if (cc < 2) cc = 2;
    while ((int64_t)cc * (cc - 1) * (cc - 2) / 6 > tt) cc--;
    while ((int64_t)(cc + 1) * cc * (cc - 1) / 6 <= tt) cc++;
    int64_t rem = tt - (int64_t)cc * (cc - 1) * (cc - 2) / 6;
    int bb_ = (int)sqrt(2.0 * (double)rem);
    if (bb_ < 1) bb_ = 1;
    while ((int64_t)bb_ * (bb_ - 1) / 2 > rem) bb_--;
    while ((int64_t)(bb_ + 1) * bb_ / 2 <= rem) bb_++;
    *aa = (int)(rem - (int64_t)bb_ * (bb_ - 1) / 2);
    *bb = bb_;
    *cc_out = cc;
}

/* type-3 decode (mc.cu:222-227) */
static void decode_pair(int64_t tt, int* aa, int* bb) {
    int bb_ = (int)sqrt(2.0 * (double)tt);
    if (bb_ < 1) bb_ = 1;
    while ((int64_t)bb_ * (bb_ - 1) / 2 > tt) bb_--;
    while ((int64_t)(bb_ + 1) * bb_ / 2 <= tt) bb_++;
    *aa = (int)(tt - (int64_t)bb_ * (bb_ - 1) / 2);
    *bb = bb_;
}

static inline int skip2(int x, int i0, int j0) {   /* mc.cu:199-201 */
    if (x >= i0) x++;
    if (x >= j0) x++;
    return x;
}

/* 3-type term t of move (i0,j0) -> sorted quartet (mc.cu:186-238) */
static void three_type_term(int64_t t, int64_t n_type12, int i0, int j0, int* idx) {
    int a, b, c;
    if (t < n_type12) {
        decode_triple(t, &a, &b, &c);
        idx[0] = i0; idx[1] = skip2(a, i0, j0); idx[2] = skip2(b, i0, j0); idx[3] = skip2(c, i0, j0);
    } else if (t < 2 * n_type12) {
        decode_triple(t - n_type12, &a, &b, &c);
        idx[0] = j0; idx[1] = skip2(a, i0, j0); idx[2] = skip2(b, i0, j0); idx[3] = skip2(c, i0, j0);
    } else {
        decode_pair(t - 2 * n_type12, &a, &b);
        idx[0] = i0; idx[1] = j0; idx[2] = skip2(a, i0, j0); idx[3] = skip2(b, i0, j0);
    }
    sort4(idx);
}

int64_t orc_three_type(int N, int i0, int j0, int32_t* out) {
    int64_t n_type12 = (int64_t)(N - 2) * (N - 3) * (N - 4) / 6;   /* mc.cu:115 */
    int64_t n_type3 = (int64_t)(N - 2) * (N - 3) / 2;               /* mc.cu:116 */
    int64_t n_h4 = 2 * n_type12 + n_type3;
    for (int64_t t = 0; t < n_h4; t++) {
        int idx[4];
        three_type_term(t, n_type12, i0, j0, idx);
        if (out) for (int p = 0; p < 4; p++) out[4 * t + p] = idx[p];
    }
    return n_h4;
}

/* ------------------------------------------------------------------ */
/* configuration                                                        */
/* ------------------------------------------------------------------ */

/* config.cu:61-67 */
double orc_auto_gamma(int fmc_mode, int N, double gamma) {
    if (fmc_mode > 0 && gamma <= 0.0) {
        if (fmc_mode == 1) return 0.0;
        if (fmc_mode == 2) return 1.0 / (2.0 * (N - 1));
    }
    return gamma;
}

/* parallel_tempering.cu:93-109 (index 0 is the hottest) */
void orc_temperature_schedule(int NT, double Tmin, double Tmax, int log_temp,
                              double* T, double* beta) {
    if (log_temp) {
        double A = (NT > 1) ? pow(Tmin / Tmax, 1.0 / (NT - 1)) : 1.0;
        for (int t = 0; t < NT; t++) { T[t] = Tmax * pow(A, t); beta[t] = 1.0 / T[t]; }
    } else {
        double dT = (NT > 1) ? (Tmax - Tmin) / (NT - 1) : 0.0;
        for (int t = 0; t < NT; t++) { T[t] = Tmax - t * dT; beta[t] = 1.0 / T[t]; }
    }
}

/* ------------------------------------------------------------------ */
/* frequencies and FMC                                                  */
/* ------------------------------------------------------------------ */

static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* mc.cu:449-460 (comb omega_k = k; uniform splitmix64(seed+3000) >> 11 / 2^53, sorted) */
void orc_omega(int N, int fmc_mode, uint64_t seed, double* omega) {
    if (fmc_mode == 1) {
        for (int i = 0; i < N; i++) omega[i] = (double)i;
    } else {
        uint64_t st = seed + 3000;
        for (int i = 0; i < N; i++) {
            uint64_t z = orc_splitmix64(&st);
            omega[i] = (double)(z >> 11) / (double)(1ULL << 53);
        }
        qsort(omega, N, sizeof(double), cmp_double);
    }
}

/* disorder.cu:130-143: zero both halves of (i<j) when |w_i - w_j| > gamma */
void orc_fmc_g2(double* g2, int N, const double* omega, double gamma) {
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) {
            double dw = fabs(omega[i] - omega[j]);
            if (dw > gamma) {
                g2[2 * (i * N + j)] = 0.0; g2[2 * (i * N + j) + 1] = 0.0;
                g2[2 * (j * N + i)] = 0.0; g2[2 * (j * N + i) + 1] = 0.0;
            }
        }
}

/* mc.cu:469-477: non-zeros over j >= i, diagonal included */
int64_t orc_count_pairs_active(const double* g2, int N) {
    int64_t n = 0;
    for (int i = 0; i < N; i++)
        for (int j = i; j < N; j++)
            if (g2[2 * (i * N + j)] != 0.0 || g2[2 * (i * N + j) + 1] != 0.0) n++;
    return n;
}

/* disorder.cu:173-180: first channel passing wins; evaluation order
 * ((w_a + w_b) - w_c) - w_d exactly as written there */
uint8_t orc_fmc_channel(int ii, int jj, int kk, int ll, const double* omega, double gamma) {
    if (fabs(omega[ii] + omega[jj] - omega[kk] - omega[ll]) <= gamma) return 1u;
    if (fabs(omega[ii] + omega[ll] - omega[jj] - omega[kk]) <= gamma) return 2u;
    if (fabs(omega[ii] + omega[kk] - omega[jj] - omega[ll]) <= gamma) return 4u;
    return 0u;
}

/* disorder.cu:153-183 */
void orc_fmc_g4_mask(uint8_t* mask, int N, const double* omega, double gamma) {
    int64_t nq = orc_n_quartets(N);
    #pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < nq; q++) {
        int i, j, k, l;
        orc_decode_quartet(q, &i, &j, &k, &l);
        mask[q] = orc_fmc_channel(i, j, k, l, omega, gamma);
    }
}

/* disorder.cu:234-243 */
int64_t orc_count_active_g4(const uint8_t* mask, int64_t nq) {
    int64_t c = 0;
    for (int64_t q = 0; q < nq; q++) c += __builtin_popcount(mask[q]);
    return c;
}

int64_t orc_count_survivors(int N, const double* omega, double gamma, int64_t* counts) {
    int64_t c0 = 0, c1 = 0, c2 = 0;
    #pragma omp parallel for schedule(dynamic, 1) reduction(+:c0,c1,c2)
    for (int l = N - 1; l >= 3; l--)
        for (int k = 2; k < l; k++)
            for (int j = 1; j < k; j++)
                for (int i = 0; i < j; i++) {
                    uint8_t m = orc_fmc_channel(i, j, k, l, omega, gamma);
                    c0 += (m == 1); c1 += (m == 2); c2 += (m == 4);
                }
    if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
    return c0 + c1 + c2;
}

/* ------------------------------------------------------------------ */
/* cuRAND host generator (library call)                                  */
/* ------------------------------------------------------------------ */

int orc_curand_normals(uint64_t seed, int64_t count, double* out) {
    curandGenerator_t g;
    if (curandCreateGeneratorHost(&g, CURAND_RNG_PSEUDO_PHILOX4_32_10) != CURAND_STATUS_SUCCESS) return 1;
    int rc = 0;
    if (curandSetPseudoRandomGeneratorSeed(g, seed) != CURAND_STATUS_SUCCESS) rc = 2;
    if (!rc && curandGenerateNormalDouble(g, out, (size_t)count, 0.0, 1.0) != CURAND_STATUS_SUCCESS) rc = 3;
    curandDestroyGenerator(g);
    return rc;
}

/* ------------------------------------------------------------------ */
/* disorder assembly                                                     */
/* ------------------------------------------------------------------ */

/* disorder.cu:57-80: unit normals -> imag zeroed -> lower <- upper, diagonal kept */
void orc_build_g2(const double* normals, int N, double* g2) {
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            int src = (i > j) ? (j * N + i) : (i * N + j);
            g2[2 * (i * N + j)] = normals[2 * src];
            g2[2 * (i * N + j) + 1] = 0.0;
        }
}

/* disorder.cu:93-113 */
void orc_build_g4(const double* normals, int64_t nq, double* g4) {
    for (int64_t q = 0; q < nq; q++) { g4[2 * q] = normals[2 * q]; g4[2 * q + 1] = 0.0; }
}

/* disorder.cu:28-35 */
void orc_scale(double* c, int64_t n, double sigma) {
    for (int64_t q = 0; q < n; q++) { c[2 * q] *= sigma; c[2 * q + 1] *= sigma; }
}

/* disorder.cu:200-208 */
void orc_shift_mean(double* c, int64_t n, double mean) {
    if (n <= 0 || mean == 0.0) return;
    for (int64_t q = 0; q < n; q++)
        if (c[2 * q] != 0.0 || c[2 * q + 1] != 0.0) c[2 * q] += mean;
}

/* ------------------------------------------------------------------ */
/* spins                                                                 */
/* ------------------------------------------------------------------ */

/* shared-memory tree of normalize_spins_kernel (spins.cu:95-104):
 * for s = bd/2 .. 1: sdata[t] += sdata[t+s] for t < s.  For bd not a power
 * of two the upper elements are dropped (the F8 truncation). */
static double tree_sum(double* sdata, int bd) {
    for (int s = bd / 2; s > 0; s >>= 1)
        for (int t = 0; t < s; t++) sdata[t] += sdata[t + s];
    return sdata[0];
}

/* spins.cu:27-69 (kernel path N <= 1024) and spins.cu:85-111 (host path) */
void orc_normalize_sphere(double* sp, int N, int exact) {
    double norm_sq = 0.0;
    if (exact || N > 1024) {
        for (int i = 0; i < N; i++) norm_sq += sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1];
    } else {
        int bd = N;   /* block_size = N for N < 1024, 1024 for N == 1024 */
        double* s = (double*)malloc(sizeof(double) * bd);
        for (int t = 0; t < bd; t++) s[t] = (t < N) ? sp[2 * t] * sp[2 * t] + sp[2 * t + 1] * sp[2 * t + 1] : 0.0;
        norm_sq = tree_sum(s, bd);
        free(s);
    }
    double scale = sqrt((double)N / norm_sq);
    for (int i = 0; i < N; i++) { sp[2 * i] *= scale; sp[2 * i + 1] *= scale; }
}

/* spins_sparse.cu:28-61 and :76 (block = round_up32(N) capped at 1024, one block) */
void orc_normalize_cube(double* sp, int N, int exact) {
    int bd = (N < 1024) ? ((N + 31) / 32 * 32) : 1024;
    if (bd < 32) bd = 32;
    double sum = 0.0;
    if (exact) {
        for (int i = 0; i < N; i++) { double r2 = sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1]; sum += r2 * r2; }
    } else {
        double* s = (double*)malloc(sizeof(double) * bd);
        for (int t = 0; t < bd; t++) {
            double r2 = (t < N) ? sp[2 * t] * sp[2 * t] + sp[2 * t + 1] * sp[2 * t + 1] : 0.0;
            s[t] = r2 * r2;
        }
        sum = tree_sum(s, bd);
        free(s);
    }
    double scale = pow((double)N / sum, 0.25);
    int lim = exact ? N : (N < bd ? N : bd);
    for (int i = 0; i < lim; i++) { sp[2 * i] *= scale; sp[2 * i + 1] *= scale; }
}

/* ------------------------------------------------------------------ */
/* complex helpers (cuCmul semantics)                                    */
/* ------------------------------------------------------------------ */
typedef struct { double x, y; } cplx;
static inline cplx cm(cplx a, cplx b) { cplx r = { a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x }; return r; }
static inline cplx cj(cplx a) { cplx r = { a.x, -a.y }; return r; }
static inline cplx ld(const double* p, int i) { cplx r = { p[2 * i], p[2 * i + 1] }; return r; }

/* mc.cu:385-395: channel term with conjugation pattern */
static inline double quartet_term(cplx gq, int ch, cplx ai, cplx aj, cplx ak, cplx al) {
    cplx s0, s1, s2, s3;
    if (ch == 0)      { s0 = ai; s1 = aj;     s2 = cj(ak); s3 = cj(al); }
    else if (ch == 1) { s0 = ai; s1 = cj(aj); s2 = cj(ak); s3 = al; }
    else              { s0 = ai; s1 = cj(aj); s2 = ak;     s3 = cj(al); }
    cplx prod = cm(gq, cm(cm(s0, s1), cm(s2, s3)));
    return -prod.x;
}

/* ------------------------------------------------------------------ */
/* energies                                                              */
/* ------------------------------------------------------------------ */

/* mc.cu:343-396 (init_energy_kernel) split as in mc.cu:567-656 */
void orc_energy_dense(int N, const double* g2, const double* g4, const uint8_t* mask,
                      int h2_active, const double* sp, double* e2, double* e4) {
    double s2 = 0.0, s4 = 0.0;
    if (h2_active)
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++) {
                cplx g = ld(g2, i * N + j);
                cplx prod = cm(g, cm(ld(sp, i), cj(ld(sp, j))));
                s2 += -prod.x;
            }
    /* quartets in q order (q = C(l,4)+C(k,3)+C(j,2)+i, i fastest), one
       partial sum per l, added in l order: deterministic for any thread count */
    double* part = (double*)calloc((size_t)(N > 0 ? N : 1), sizeof(double));
    #pragma omp parallel for schedule(dynamic, 1)
    for (int l = 3; l < N; l++) {
        double t = 0.0;
        int64_t q = orc_n_quartets(l);
        for (int k = 2; k < l; k++)
            for (int j = 1; j < k; j++)
                for (int i = 0; i < j; i++, q++) {
                    cplx gq = { g4[2 * q], g4[2 * q + 1] };
                    uint8_t m = mask[q];
                    if ((gq.x == 0.0 && gq.y == 0.0) || m == 0) continue;
                    for (int ch = 0; ch < 3; ch++)
                        if (m & (1 << ch)) t += quartet_term(gq, ch, ld(sp, i), ld(sp, j), ld(sp, k), ld(sp, l));
                }
        part[l] = t;
    }
    for (int l = 3; l < N; l++) s4 += part[l];
    free(part);
    if (e2) *e2 = s2;
    if (e4) *e4 = s4;
}

/* mc_sparse.cu:277-306 */
void orc_energy_sparse(int N, const double* g2, int nq, const int32_t* Q, const double* qg,
                       int h2_active, const double* sp, double* e2, double* e4) {
    double s2 = 0.0, s4 = 0.0;
    if (h2_active)
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++) {
                cplx g = ld(g2, i * N + j);
                cplx prod = cm(g, cm(ld(sp, i), cj(ld(sp, j))));
                s2 += -prod.x;
            }
    for (int q = 0; q < nq; q++) {
        cplx gq = { qg[q], 0.0 };
        const int32_t* e = Q + 5 * q;
        s4 += quartet_term(gq, e[4], ld(sp, e[0]), ld(sp, e[1]), ld(sp, e[2]), ld(sp, e[3]));
    }
    if (e2) *e2 = s2;
    if (e4) *e4 = s4;
}

/* hamiltonian.cu:23-58: H2 over i <= j, diagonal included */
double orc_energy_h2_with_diag(int N, const double* g2, const double* sp) {
    double s = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = i; j < N; j++) {
            cplx prod = cm(ld(g2, i * N + j), cm(ld(sp, i), cj(ld(sp, j))));
            s += -prod.x;
        }
    return s;
}

static double abs_h2(int N, const double* g2, const double* so, const double* sn, int i0, int j0) {
    double s = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) {
            if (i != i0 && i != j0 && j != i0 && j != j0) continue;
            cplx g = ld(g2, i * N + j);
            s += fabs(cm(g, cm(ld(so, i), cj(ld(so, j)))).x);
            s += fabs(cm(g, cm(ld(sn, i), cj(ld(sn, j)))).x);
        }
    return s;
}

double orc_dense_abs_terms(int N, const double* g2, const double* g4, const uint8_t* mask,
                           int h2_active, const double* so, const double* sn, int i0, int j0) {
    double s = h2_active ? abs_h2(N, g2, so, sn, i0, j0) : 0.0;
    /* quartets in q order; only those holding i0 or j0 contribute */
    int64_t q = 0;
    for (int l = 3; l < N; l++)
        for (int k = 2; k < l; k++)
            for (int j = 1; j < k; j++) {
                const int hit_jkl = (j == i0 || j == j0 || k == i0 || k == j0 || l == i0 || l == j0);
                for (int i = 0; i < j; i++, q++) {
                    if (!hit_jkl && i != i0 && i != j0) continue;
                    uint8_t m = mask[q];
                    cplx gq = { g4[2 * q], g4[2 * q + 1] };
                    if ((gq.x == 0.0 && gq.y == 0.0) || m == 0) continue;
                    for (int ch = 0; ch < 3; ch++)
                        if (m & (1 << ch)) {
                            s += fabs(quartet_term(gq, ch, ld(so, i), ld(so, j), ld(so, k), ld(so, l)));
                            s += fabs(quartet_term(gq, ch, ld(sn, i), ld(sn, j), ld(sn, k), ld(sn, l)));
                        }
                }
            }
    return s;
}

double orc_sparse_abs_terms(int N, const double* g2, int nq, const int32_t* Q, const double* qg,
                            int h2_active, const double* so, const double* sn, int i0, int j0) {
    double s = h2_active ? abs_h2(N, g2, so, sn, i0, j0) : 0.0;
    for (int q = 0; q < nq; q++) {
        const int32_t* e = Q + 5 * q;
        int touch = 0;
        for (int p = 0; p < 4; p++) touch |= (e[p] == i0 || e[p] == j0);
        if (!touch) continue;
        cplx gq = { qg[q], 0.0 };
        s += fabs(quartet_term(gq, e[4], ld(so, e[0]), ld(so, e[1]), ld(so, e[2]), ld(so, e[3])));
        s += fabs(quartet_term(gq, e[4], ld(sn, e[0]), ld(sn, e[1]), ld(sn, e[2]), ld(sn, e[3])));
    }
    return s;
}

/* ------------------------------------------------------------------ */
/* init (mc_init / mc_sparse_init)                                       */
/* ------------------------------------------------------------------ */

static void split_J(const orc_config* c, double* J2, double* J4, double* J20, double* J40) {
    *J2 = (1.0 - c->alpha) * c->J;      /* mc.cu:436-439 */
    *J4 = c->alpha * c->J;
    *J20 = (1.0 - c->alpha0) * c->J0;
    *J40 = c->alpha0 * c->J0;
}

/* g2 generation + FMC + count + rescale + mean shift; shared by both variants
 * (mc.cu:443-498, mc_sparse.cu:422-475).  Returns omega filled when fmc>0. */
static int g2_and_omega(const orc_config* c, double* g2, double* omega, int64_t* n_pairs_active) {
    int N = c->N;
    double J2, J4, J20, J40;
    split_J(c, &J2, &J4, &J20, &J40);
    memset(g2, 0, sizeof(double) * 2 * (size_t)N * N);
    if (c->fmc_mode != 1) {
        double* nrm = (double*)malloc(sizeof(double) * 2 * (size_t)N * N);
        if (orc_curand_normals(c->seed + 1000, 2 * (int64_t)N * N, nrm)) { free(nrm); return 1; }
        orc_build_g2(nrm, N, g2);
        free(nrm);
    }
    double gamma = c->gamma;
    if (c->fmc_mode > 0) {
        orc_omega(N, c->fmc_mode, c->seed, omega);
        if (c->fmc_mode == 1) *n_pairs_active = 0;
        else {
            orc_fmc_g2(g2, N, omega, gamma);
            *n_pairs_active = orc_count_pairs_active(g2, N);
        }
    } else {
        *n_pairs_active = orc_n_pairs(N);
    }
    if (*n_pairs_active > 0) orc_scale(g2, (int64_t)N * N, J2 * sqrt((double)N / (double)*n_pairs_active));
    if (J20 != 0.0 && *n_pairs_active > 0)
        orc_shift_mean(g2, (int64_t)N * N, J20 * (double)N / (double)*n_pairs_active);
    return 0;
}

int orc_init_dense(const orc_config* c, int init_exact, double* g2, double* g4, uint8_t* mask,
                   double* omega, double* spins, double* energies, orc_disorder_info* info) {
    int N = c->N, nrep = c->nrep;
    int64_t nq = orc_n_quartets(N);
    double J2, J4, J20, J40;
    split_J(c, &J2, &J4, &J20, &J40);
    double* om = omega ? omega : (double*)malloc(sizeof(double) * N);
    int64_t npa = 0;
    if (g2_and_omega(c, g2, om, &npa)) return 1;
    double* nrm = (double*)malloc(sizeof(double) * 2 * (size_t)nq);
    if (orc_curand_normals(c->seed + 2000 + 12345, 2 * nq, nrm)) { free(nrm); return 1; }
    orc_build_g4(nrm, nq, g4);
    free(nrm);
    memset(mask, 1, (size_t)nq);                       /* init_g4_mask: 0x1 */
    int64_t nqa;
    if (c->fmc_mode > 0) {
        orc_fmc_g4_mask(mask, N, om, c->gamma);
        nqa = orc_count_active_g4(mask, nq);
    } else {
        nqa = nq;
    }
    if (nqa > 0) orc_scale(g4, nq, J4 * sqrt((double)N / (double)nqa));   /* disorder.cu:115-124 */
    if (J40 != 0.0 && nqa > 0) orc_shift_mean(g4, nq, J40 * (double)N / (double)nqa);
    int h2 = npa > 0;
    uint64_t* seeds = (uint64_t*)malloc(sizeof(uint64_t) * nrep);
    orc_replica_seeds(c->seed, nrep, seeds);
    for (int r = 0; r < nrep; r++) {
        double* sp = spins + 2 * (size_t)r * N;
        if (orc_curand_normals(seeds[r], 2 * (int64_t)N, sp)) { free(seeds); return 1; }
        orc_normalize_sphere(sp, N, init_exact);
    }
    free(seeds);
    if (energies)
        for (int r = 0; r < nrep; r++) {
            double e2, e4;
            orc_energy_dense(N, g2, g4, mask, h2, spins + 2 * (size_t)r * N, &e2, &e4);
            energies[r] = e2 + e4;
        }
    if (info) { info->n_pairs_active = npa; info->n_quart_active = nqa; info->h2_active = h2; info->n_sparse = 0; }
    if (!omega) free(om);
    return 0;
}

/* mc_sparse.cu:340-349 (note the (int)count cast, kept) */
void orc_partial_shuffle(int64_t* arr, int64_t count, int n_select, uint64_t seed) {
    uint64_t rng = seed;
    for (int i = 0; i < n_select && i < (int)count; i++) {
        uint64_t r = orc_splitmix64(&rng);
        int64_t j = i + (int64_t)(r % (uint64_t)(count - i));
        int64_t t = arr[i]; arr[i] = arr[j]; arr[j] = t;
    }
}

int orc_sparse_select(int N, const double* omega, double gamma, int fmc_mode, uint64_t seed,
                      int n_select, int64_t* out_enc, int64_t* n_nonzero) {
    /* survivors in ascending q*3+ch order (mc_sparse.cu:491-500).  The g4
     * value test (:495) never removes anything: unit normals are never 0. */
    int64_t cap = 0, n = 0;
    int64_t* arr = NULL;
    if (fmc_mode == 0) cap = orc_n_quartets(N);
    else cap = orc_count_survivors(N, omega, gamma, NULL);
    arr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(cap > 0 ? cap : 1));
    if (!arr) return 1;
    int64_t q = 0;
    for (int l = 3; l < N; l++)
        for (int k = 2; k < l; k++)
            for (int j = 1; j < k; j++)
                for (int i = 0; i < j; i++, q++) {
                    uint8_t m = (fmc_mode == 0) ? 1u : orc_fmc_channel(i, j, k, l, omega, gamma);
                    for (int ch = 0; ch < 3; ch++)
                        if (m & (1 << ch)) arr[n++] = q * 3 + ch;
                }
    *n_nonzero = n;
    int ns = n_select;
    if (n < ns) ns = (int)n;
    orc_partial_shuffle(arr, n, ns, seed + 4000);
    for (int s = 0; s < ns; s++) out_enc[s] = arr[s];
    free(arr);
    return 0;
}

int orc_init_sparse(const orc_config* c, int init_exact, double* g2, int32_t* Q, double* qg,
                    double* omega, double* spins, double* energies, orc_disorder_info* info) {
    int N = c->N, nrep = c->nrep;
    int64_t nq = orc_n_quartets(N);
    double J2, J4, J20, J40;
    split_J(c, &J2, &J4, &J20, &J40);
    double* om = omega ? omega : (double*)malloc(sizeof(double) * N);
    int64_t npa = 0;
    if (g2_and_omega(c, g2, om, &npa)) return 1;
    int h2 = npa > 0;
    double* nrm = (double*)malloc(sizeof(double) * 2 * (size_t)nq);
    if (orc_curand_normals(c->seed + 2000 + 12345, 2 * nq, nrm)) { free(nrm); return 1; }
    int64_t* enc = (int64_t*)malloc(sizeof(int64_t) * N);
    int64_t nnz = 0;
    orc_sparse_select(N, om, c->gamma, c->fmc_mode, c->seed, N, enc, &nnz);
    int ns = (nnz < N) ? (int)nnz : N;
    double sigma = J4 * sqrt((double)N / (double)ns);                       /* mc_sparse.cu:518 */
    double mean4 = (J40 != 0.0) ? J40 * (double)N / (double)ns : 0.0;       /* :520 */
    for (int s = 0; s < ns; s++) {
        int64_t q = enc[s] / 3;
        int ch = (int)(enc[s] % 3);
        int i, j, k, l;
        orc_decode_quartet(q, &i, &j, &k, &l);
        Q[5 * s] = i; Q[5 * s + 1] = j; Q[5 * s + 2] = k; Q[5 * s + 3] = l; Q[5 * s + 4] = ch;
        qg[s] = nrm[2 * q] * sigma + mean4;                                  /* :536 */
    }
    free(nrm);
    free(enc);
    uint64_t* seeds = (uint64_t*)malloc(sizeof(uint64_t) * nrep);
    orc_replica_seeds(c->seed, nrep, seeds);
    for (int r = 0; r < nrep; r++) {
        double* sp = spins + 2 * (size_t)r * N;
        if (orc_curand_normals(seeds[r], 2 * (int64_t)N, sp)) { free(seeds); return 1; }
        orc_normalize_cube(sp, N, init_exact);
    }
    free(seeds);
    if (energies)
        for (int r = 0; r < nrep; r++) {
            double e2, e4;
            orc_energy_sparse(N, g2, ns, Q, qg, h2, spins + 2 * (size_t)r * N, &e2, &e4);
            energies[r] = e2 + e4;
        }
    if (info) { info->n_pairs_active = npa; info->n_quart_active = nnz; info->h2_active = h2; info->n_sparse = ns; }
    if (!omega) free(om);
    return 0;
}

/* ------------------------------------------------------------------ */
/* proposals                                                             */
/* ------------------------------------------------------------------ */

/* spins.h:17-52 */
void orc_propose_sphere(const double* ai, const double* aj, double u_alpha, double u_phi1,
                        double u_phi2, double* ain, double* ajn) {
    double alpha = 2.0 * M_PI * u_alpha, phi1 = 2.0 * M_PI * u_phi1, phi2 = 2.0 * M_PI * u_phi2;
    double ca = cos(alpha), sa = sin(alpha), cp1 = cos(phi1), sp1 = sin(phi1), cp2 = cos(phi2), sp2 = sin(phi2);
    double x1 = ai[0], y1 = ai[1], x2 = aj[0], y2 = aj[1];
    double r1 = x1 * x1 + y1 * y1, r2 = x2 * x2 + y2 * y2;
    double nx1 = x1 * cp1 + y1 * sp1, ny1 = -x1 * sp1 + y1 * cp1;
    double nx2 = x2 * cp2 + y2 * sp2, ny2 = -x2 * sp2 + y2 * cp2;
    double f1 = sqrt((r1 + r2) / r1) * ca, f2 = sqrt((r1 + r2) / r2) * sa;
    ain[0] = nx1 * f1; ain[1] = ny1 * f1; ajn[0] = nx2 * f2; ajn[1] = ny2 * f2;
}

/* spins_sparse.h:26-56 */
void orc_propose_cube(const double* ai, const double* aj, double u, double u_phi1, double u_phi2,
                      double* ain, double* ajn) {
    double phi1 = u_phi1 * 2.0 * M_PI, phi2 = u_phi2 * 2.0 * M_PI;
    double r1 = ai[0] * ai[0] + ai[1] * ai[1], r2 = aj[0] * aj[0] + aj[1] * aj[1];
    double S4 = r1 * r1 + r2 * r2, sS4 = sqrt(S4);
    double m1 = sqrt(sS4 * sqrt(1.0 - u)), m2 = sqrt(sS4 * sqrt(u));
    ain[0] = m1 * cos(phi1); ain[1] = m1 * sin(phi1);
    ajn[0] = m2 * cos(phi2); ajn[1] = m2 * sin(phi2);
}

/* ------------------------------------------------------------------ */
/* random streams                                                        */
/* ------------------------------------------------------------------ */

/* Philox4x32-10 (Salmon et al., SC'11): round
 *   (hi0,lo0) = M0*c0, (hi1,lo1) = M1*c2,
 *   c <- (hi1^c1^k0, lo1, hi0^c3^k1, lo0); key bumped by the Weyl constants. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* POSIX srand48: high 32 bits of X from the seed, low 16 bits 0x330E */
uint64_t orc_srand48_state(long seedval) {
    return (((uint64_t)(uint32_t)seedval) << 16) | 0x330Eu;
}

double orc_drand48(uint64_t* st) {
    *st = (0x5DEECE66DULL * *st + 0xBULL) & 0xFFFFFFFFFFFFULL;
    return (double)*st * (1.0 / 281474976710656.0);
}

/* ------------------------------------------------------------------ */
/* replica exchange (parallel_tempering.cu:316-352)                     */
/* ------------------------------------------------------------------ */
void orc_exchange(int NT, int nrep, const double* bs, const double* E, int32_t* perm,
                  uint64_t* dst, int64_t* ex_acc, int64_t* ex_prop, double* betas_out) {
    for (int t = 0; t < NT - 1; t++)
        for (int r = 0; r < nrep; r++) {
            int a = perm[t * nrep + r], b = perm[(t + 1) * nrep + r];
            double delta = (bs[t] - bs[t + 1]) * (E[a] - E[b]);
            if (ex_prop) ex_prop[t]++;
            int acc = (delta >= 0.0);
            if (!acc) acc = (orc_drand48(dst) < exp(delta));
            if (acc) {
                if (ex_acc) ex_acc[t]++;
                int tmp = perm[t * nrep + r];
                perm[t * nrep + r] = perm[(t + 1) * nrep + r];
                perm[(t + 1) * nrep + r] = tmp;
            }
        }
    if (betas_out)
        for (int t = 0; t < NT; t++)
            for (int r = 0; r < nrep; r++) betas_out[perm[t * nrep + r]] = bs[t];
}

/* ------------------------------------------------------------------ */
/* CPU sweep                                                             */
/* ------------------------------------------------------------------ */

static inline double u53(uint32_t a, uint32_t b) {
    return (double)(((uint64_t)a << 21) ^ (uint64_t)(b >> 11)) * (1.0 / 9007199254740992.0);
}

typedef struct { uint32_t w[8]; int used; uint64_t key; uint64_t ctr; } orc_rng;

static void rng_refill(orc_rng* g) {
    uint32_t key[2] = { (uint32_t)g->key, (uint32_t)(g->key >> 32) };
    uint32_t c0[4] = { (uint32_t)g->ctr, (uint32_t)(g->ctr >> 32), 0u, 0x6f726331u };
    uint32_t c1[4] = { (uint32_t)g->ctr, (uint32_t)(g->ctr >> 32), 1u, 0x6f726331u };
    orc_philox4x32_10(c0, key, g->w);
    orc_philox4x32_10(c1, key, g->w + 4);
    g->ctr++;
    g->used = 0;
}

static double rng_u(orc_rng* g) {
    if (g->used > 6) rng_refill(g);
    double u = u53(g->w[g->used], g->w[g->used + 1]);
    g->used += 2;
    return u;
}

/* dense dE for move (i0,j0): H2 factored (mc.cu:161-180), H4 3-type
 * enumeration with full old/new products (mc.cu:183-275) */
static double dense_dE(const orc_sweep_args* a, const double* sp, int i0, int j0, cplx ain, cplx ajn) {
    int N = a->N;
    cplx aio = ld(sp, i0), ajo = ld(sp, j0);
    cplx di = { ain.x - aio.x, ain.y - aio.y }, dj = { ajn.x - ajo.x, ajn.y - ajo.y };
    double dE = 0.0;
    if (a->h2_active) {
        cplx si = { 0, 0 }, sj = { 0, 0 };
        for (int k = 0; k < N; k++) {
            if (k == i0 || k == j0) continue;
            cplx akc = cj(ld(sp, k));
            cplx t1 = cm(ld(a->g2, i0 * N + k), akc), t2 = cm(ld(a->g2, j0 * N + k), akc);
            si.x += t1.x; si.y += t1.y; sj.x += t2.x; sj.y += t2.y;
        }
        dE -= cm(di, si).x;
        dE -= cm(dj, sj).x;
        cplx gij = ld(a->g2, i0 * N + j0);
        cplx op = cm(gij, cm(aio, cj(ajo))), np = cm(gij, cm(ain, cj(ajn)));
        dE -= (np.x - op.x);
    }
    int64_t n_type12 = (int64_t)(N - 2) * (N - 3) * (N - 4) / 6;
    int64_t n_h4 = 2 * n_type12 + (int64_t)(N - 2) * (N - 3) / 2;
    static const int conj_masks[3] = { 0xC, 0x6, 0xA };
    for (int64_t t = 0; t < n_h4; t++) {
        int idx[4];
        three_type_term(t, n_type12, i0, j0, idx);
        int64_t q = orc_encode_quartet(idx[0], idx[1], idx[2], idx[3]);
        cplx gq = { a->g4[2 * q], a->g4[2 * q + 1] };
        uint8_t qm = a->mask[q];
        if ((gq.x == 0.0 && gq.y == 0.0) || qm == 0) continue;
        for (int ch = 0; ch < 3; ch++) {
            if (!(qm & (1 << ch))) continue;
            int cmk = conj_masks[ch];
            cplx of[4], nf[4];
            for (int p = 0; p < 4; p++) {
                cplx ov = ld(sp, idx[p]), nv = ov;
                if (idx[p] == i0) nv = ain; else if (idx[p] == j0) nv = ajn;
                of[p] = ((cmk >> p) & 1) ? cj(ov) : ov;
                nf[p] = ((cmk >> p) & 1) ? cj(nv) : nv;
            }
            cplx opr = cm(gq, cm(cm(of[0], of[1]), cm(of[2], of[3])));
            cplx npr = cm(gq, cm(cm(nf[0], nf[1]), cm(nf[2], nf[3])));
            dE -= (npr.x - opr.x);
        }
    }
    return dE;
}

/* sparse dE (mc_sparse.cu:146-210) */
static double sparse_dE(const orc_sweep_args* a, const double* sp, int i0, int j0, cplx ain, cplx ajn) {
    int N = a->N;
    cplx aio = ld(sp, i0), ajo = ld(sp, j0);
    cplx di = { ain.x - aio.x, ain.y - aio.y }, dj = { ajn.x - ajo.x, ajn.y - ajo.y };
    double dE = 0.0;
    if (a->h2_active) {
        cplx si = { 0, 0 }, sj = { 0, 0 };
        for (int k = 0; k < N; k++) {
            if (k == i0 || k == j0) continue;
            cplx akc = cj(ld(sp, k));
            cplx t1 = cm(ld(a->g2, i0 * N + k), akc), t2 = cm(ld(a->g2, j0 * N + k), akc);
            si.x += t1.x; si.y += t1.y; sj.x += t2.x; sj.y += t2.y;
        }
        dE -= cm(di, si).x;
        dE -= cm(dj, sj).x;
        cplx gij = ld(a->g2, i0 * N + j0);
        cplx op = cm(gij, cm(aio, cj(ajo))), np = cm(gij, cm(ain, cj(ajn)));
        dE -= (np.x - op.x);
    }
    static const int conj_masks[3] = { 0xC, 0x6, 0xA };
    for (int q = 0; q < a->nq; q++) {
        const int32_t* e = a->q_ijklch + 5 * q;
        int inv_i = (e[0] == i0 || e[1] == i0 || e[2] == i0 || e[3] == i0);
        int inv_j = (e[0] == j0 || e[1] == j0 || e[2] == j0 || e[3] == j0);
        if (!inv_i && !inv_j) continue;
        int cmk = conj_masks[e[4]];
        cplx g = { a->q_g[q], 0.0 };
        if (inv_i && inv_j) {
            cplx of[4], nf[4];
            for (int p = 0; p < 4; p++) {
                cplx ov = ld(sp, e[p]), nv = ov;
                if (e[p] == i0) nv = ain; else if (e[p] == j0) nv = ajn;
                of[p] = ((cmk >> p) & 1) ? cj(ov) : ov;
                nf[p] = ((cmk >> p) & 1) ? cj(nv) : nv;
            }
            cplx opr = cm(g, cm(cm(of[0], of[1]), cm(of[2], of[3])));
            cplx npr = cm(g, cm(cm(nf[0], nf[1]), cm(nf[2], nf[3])));
            dE -= (npr.x - opr.x);
        } else {
            int changed = inv_i ? i0 : j0;
            cplx d = (changed == i0) ? di : dj;
            cplx f[4];
            for (int p = 0; p < 4; p++) {
                cplx b = (e[p] == changed) ? d : ld(sp, e[p]);
                f[p] = ((cmk >> p) & 1) ? cj(b) : b;
            }
            dE -= cm(g, cm(cm(f[0], f[1]), cm(f[2], f[3]))).x;
        }
    }
    return dE;
}

void orc_sweep(orc_sweep_args* a, int nsweeps) {
    int N = a->N;
#ifdef _OPENMP
    int nt = a->nthreads > 0 ? a->nthreads : omp_get_max_threads();
#endif
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int r = 0; r < a->nrep; r++) {
        double* sp = a->spins + 2 * (size_t)r * N;
        orc_rng g;
        g.key = a->seeds[r]; g.ctr = a->move_counter[r]; g.used = 8;
        double E = a->energies[r], beta = a->betas[r];
        int64_t acc = 0, prop = 0;
        for (int s = 0; s < nsweeps; s++)
            for (int step = 0; step < N / 2; step++) {
                int ri = (int)(rng_u(&g) * N);            /* mc.cu:131-139 */
                if (ri >= N) ri = N - 1;
                int rj = (int)(rng_u(&g) * (N - 1));
                if (rj >= N - 1) rj = N - 2;
                if (rj >= ri) rj++;
                int i0 = ri < rj ? ri : rj, j0 = ri < rj ? rj : ri;
                double ain[2], ajn[2];
                double u1 = rng_u(&g), u2 = rng_u(&g), u3 = rng_u(&g);
                if (a->variant == 0) orc_propose_sphere(sp + 2 * i0, sp + 2 * j0, u1, u2, u3, ain, ajn);
                else orc_propose_cube(sp + 2 * i0, sp + 2 * j0, u1, u2, u3, ain, ajn);
                cplx ci = { ain[0], ain[1] }, cjn = { ajn[0], ajn[1] };
                prop++;
                double dE = (a->variant == 0) ? dense_dE(a, sp, i0, j0, ci, cjn)
                                              : sparse_dE(a, sp, i0, j0, ci, cjn);
                int accept;                                 /* mc.cu:288-297 */
                if (beta == 0.0) accept = 1;
                else {
                    accept = (dE <= 0.0);
                    if (!accept) accept = (rng_u(&g) < exp(-beta * dE));
                }
                if (accept) {
                    sp[2 * i0] = ain[0]; sp[2 * i0 + 1] = ain[1];
                    sp[2 * j0] = ajn[0]; sp[2 * j0 + 1] = ajn[1];
                    E += dE;
                    acc++;
                }
            }
        a->energies[r] = E;
        a->accepted[r] += acc;
        a->proposed[r] += prop;
        a->move_counter[r] = g.ctr;
    }
}
