// analysis.cu -- overlap histograms of saved configurations on the GPU: the
// hot loops of the reference's analysis_pt.cpp for the Parisi P(q)
// (:1337-1437), the intensity fluctuation overlap IFO (:1498-1619), the
// experimental IFO of time-averaged spectra (:1679-1806), the deeper block's
// P(|a|^2), inverse participation ratios, phase and link overlaps and
// q-q_link scatter (:1871-2045) and the multi-overlap scatter (:3468-3643).
//
// configs: [nsnap][NT][nrep][N][2] doubles (the body of configs.bin without
// the per-snapshot sweep numbers).  One thread per (snapshot, temperature,
// replica pair a < b): q = Re sum_k a_k conj(b_k) / N summed over k in order
// with round-to-nearest products and sums, no contraction, like the
// reference's loop, so every q falls in the same bin:
// bin = (int)((q - qmin) / dq), clamped to [0, nbins).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace pspin {

__global__ void overlap_count_kernel(const double* __restrict__ cfg, int N, int NT, int nrep, int nsnap, int nbins,
                                     double qmin, double dq, unsigned long long* __restrict__ counts) {
    const int npairs = nrep * (nrep - 1) / 2;
    const long long total = (long long)nsnap * NT * npairs;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int pr = (int)(id % npairs);
        const int t = (int)((id / npairs) % NT);
        const long long sn = id / ((long long)npairs * NT);
        int a = 0, rem = pr;
        while (rem >= nrep - 1 - a) { rem -= nrep - 1 - a; a++; }
        const int b = a + 1 + rem;
        const double* x = cfg + ((sn * NT + t) * nrep + a) * 2LL * N;
        const double* y = cfg + ((sn * NT + t) * nrep + b) * 2LL * N;
        double s = 0.0;
        for (int k = 0; k < N; k++)
            s = __dadd_rn(s, __dadd_rn(__dmul_rn(x[2 * k], y[2 * k]), __dmul_rn(x[2 * k + 1], y[2 * k + 1])));
        const double q = __ddiv_rn(s, (double)N);
        int bin = (int)__ddiv_rn(__dsub_rn(q, qmin), dq);
        if (bin < 0) bin = 0;
        if (bin >= nbins) bin = nbins - 1;
        atomicAdd(counts + (size_t)t * nbins + bin, 1ull);
    }
}

// ---- intensity fluctuation overlaps ----------------------------------------
// I_k = |a_k|^2 of a saved configuration, <I_k>_r its mean over the nsnap
// snapshots of one replica (summed in snapshot order, then divided), all in
// round-to-nearest FP64 operations without contraction in the reference's
// order, so every overlap C lands in the reference's bin.  Pairs whose norm
// product is not positive are skipped and not counted (the reference's
// `den <= 0` case); n_valid[t] counts the others.
__device__ __forceinline__ double intensity(const double* x, int k) {
    return __dadd_rn(__dmul_rn(x[2 * k], x[2 * k]), __dmul_rn(x[2 * k + 1], x[2 * k + 1]));
}

__device__ __forceinline__ void count_overlap(double num, double den, int nbins, double cmin, double dc,
                                              unsigned long long* counts, unsigned long long* n_valid) {
    if (den <= 0.0) return;
    const double C = __ddiv_rn(num, den);
    int bin = (int)__ddiv_rn(__dsub_rn(C, cmin), dc);
    if (bin < 0) bin = 0;
    if (bin >= nbins) bin = nbins - 1;
    atomicAdd(counts + bin, 1ull);
    atomicAdd(n_valid, 1ull);
}

// meanI[t][r][k], one thread per (t, r, k)
__global__ void intensity_mean_kernel(const double* __restrict__ cfg, int N, int NT, int nrep, int nsnap,
                                      double* __restrict__ meanI) {
    const long long total = (long long)NT * nrep * N;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(id % N);
        const long long tr = id / N;                       // t * nrep + r
        double s = 0.0;
        for (int sn = 0; sn < nsnap; sn++) s = __dadd_rn(s, intensity(cfg + ((long long)sn * NT * nrep + tr) * 2LL * N, k));
        meanI[id] = __ddiv_rn(s, (double)nsnap);
    }
}

// norm2[sn][t][r] = sum_k (I_k - <I_k>_r)^2, one thread per (sn, t, r)
__global__ void ifo_norm_kernel(const double* __restrict__ cfg, const double* __restrict__ meanI, int N, int NT,
                                int nrep, int nsnap, double* __restrict__ norm2) {
    const long long total = (long long)nsnap * NT * nrep;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const long long tr = id % ((long long)NT * nrep);
        const double* x = cfg + id * 2LL * N;
        const double* m = meanI + tr * N;
        double s = 0.0;
        for (int k = 0; k < N; k++) {
            const double d = __dsub_rn(intensity(x, k), m[k]);
            s = __dadd_rn(s, __dmul_rn(d, d));
        }
        norm2[id] = s;
    }
}

// one thread per (snapshot, temperature, replica pair a < b)
__global__ void ifo_count_kernel(const double* __restrict__ cfg, const double* __restrict__ meanI,
                                 const double* __restrict__ norm2, int N, int NT, int nrep, int nsnap, int nbins,
                                 double cmin, double dc, unsigned long long* __restrict__ counts,
                                 unsigned long long* __restrict__ n_valid) {
    const int npairs = nrep * (nrep - 1) / 2;
    const long long total = (long long)nsnap * NT * npairs;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int pr = (int)(id % npairs);
        const int t = (int)((id / npairs) % NT);
        const long long sn = id / ((long long)npairs * NT);
        int a = 0, rem = pr;
        while (rem >= nrep - 1 - a) { rem -= nrep - 1 - a; a++; }
        const int b = a + 1 + rem;
        const long long ia = (sn * NT + t) * nrep + a, ib = (sn * NT + t) * nrep + b;
        const double den = __dsqrt_rn(__dmul_rn(norm2[ia], norm2[ib]));
        const double* x = cfg + ia * 2LL * N;
        const double* y = cfg + ib * 2LL * N;
        const double* ma = meanI + ((long long)t * nrep + a) * N;
        const double* mb = meanI + ((long long)t * nrep + b) * N;
        double num = 0.0;
        for (int k = 0; k < N; k++)
            num = __dadd_rn(num, __dmul_rn(__dsub_rn(intensity(x, k), ma[k]), __dsub_rn(intensity(y, k), mb[k])));
        count_overlap(num, den, nbins, cmin, dc, counts + (size_t)t * nbins, n_valid + t);
    }
}

// experimental IFO: delta_k^r = <I_k>_r - <<I_k>> with <<I_k>> the replica
// mean of <I_k>_r; one overlap per (temperature, pair), one thread each
__global__ void exp_ifo_count_kernel(const double* __restrict__ meanI, int N, int NT, int nrep, int nbins,
                                     double cmin, double dc, unsigned long long* __restrict__ counts,
                                     unsigned long long* __restrict__ n_valid) {
    const int npairs = nrep * (nrep - 1) / 2;
    const long long total = (long long)NT * npairs;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int pr = (int)(id % npairs);
        const int t = (int)(id / npairs);
        int a = 0, rem = pr;
        while (rem >= nrep - 1 - a) { rem -= nrep - 1 - a; a++; }
        const int b = a + 1 + rem;
        const double* m = meanI + (long long)t * nrep * N;
        double na = 0.0, nb = 0.0, num = 0.0;
        for (int k = 0; k < N; k++) {
            double g = 0.0;
            for (int r = 0; r < nrep; r++) g = __dadd_rn(g, m[(long long)r * N + k]);
            g = __ddiv_rn(g, (double)nrep);
            const double da = __dsub_rn(m[(long long)a * N + k], g), db = __dsub_rn(m[(long long)b * N + k], g);
            na = __dadd_rn(na, __dmul_rn(da, da));
            nb = __dadd_rn(nb, __dmul_rn(db, db));
            num = __dadd_rn(num, __dmul_rn(da, db));
        }
        count_overlap(num, __dsqrt_rn(__dmul_rn(na, nb)), nbins, cmin, dc, counts + (size_t)t * nbins, n_valid + t);
    }
}


// ---- the deeper block of analysis_pt.cpp (:1871-2045) ---------------------
// Per configuration (snapshot, temperature, replica): the intensities
// I_k = re^2 + im^2 binned for P(|a|^2) (bin = (int)(I_k / da2), kept when in
// [0, nbins_a2)) and the inverse participation terms sum I^2 / (sum I)^2 and
// sum I^4 / (sum I)^4, the sums taken over k in order (I^4 as ((I I) I) I).
// y[.][0..2] = Y2 term, Y4 term, 1 when (sum I)^2 > 0 (else the terms are 0
// and the configuration is not counted).
__global__ void deep_site_kernel(const double* __restrict__ cfg, int N, int NT, int nrep, int nsnap, int nbins_a2,
                                 double da2, unsigned long long* __restrict__ marg, double* __restrict__ y) {
    const long long total = (long long)nsnap * NT * nrep;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int t = (int)((id / nrep) % NT);
        const double* x = cfg + id * 2LL * N;              // [sn][t][r] is row id
        double sI = 0.0, sI2 = 0.0, sI4 = 0.0;
        for (int k = 0; k < N; k++) {
            const double Ik = intensity(x, k);
            const double Ik2 = __dmul_rn(Ik, Ik);
            sI = __dadd_rn(sI, Ik);
            sI2 = __dadd_rn(sI2, Ik2);
            sI4 = __dadd_rn(sI4, __dmul_rn(__dmul_rn(Ik2, Ik), Ik));
            const int bin = (int)__ddiv_rn(Ik, da2);
            if (bin >= 0 && bin < nbins_a2) atomicAdd(marg + (size_t)t * nbins_a2 + bin, 1ull);
        }
        const double d2 = __dmul_rn(sI, sI);
        double* o = y + id * 3;
        if (d2 > 0.0) {
            o[0] = __ddiv_rn(sI2, d2);
            o[1] = __ddiv_rn(sI4, __dmul_rn(d2, d2));
            o[2] = 1.0;
        } else {
            o[0] = o[1] = o[2] = 0.0;
        }
    }
}

// Re of a quartet's product with its channel's conjugations
// (analysis_pt.cpp:334-347), round-to-nearest without contraction.
__device__ __forceinline__ double link_term(const double* d, const int* q) {
    const double ri = d[2 * q[0]], rj = d[2 * q[1]], rk = d[2 * q[2]], rl = d[2 * q[3]];
    double xi = d[2 * q[0] + 1], xj = d[2 * q[1] + 1], xk = d[2 * q[2] + 1], xl = d[2 * q[3] + 1];
    const int ch = q[4];
    if (ch == 0) { xk = -xk; xl = -xl; }
    else if (ch == 1) { xj = -xj; xk = -xk; }
    else { xj = -xj; xl = -xl; }
    const double p01r = __dsub_rn(__dmul_rn(ri, rj), __dmul_rn(xi, xj));
    const double p01i = __dadd_rn(__dmul_rn(ri, xj), __dmul_rn(xi, rj));
    const double p23r = __dsub_rn(__dmul_rn(rk, rl), __dmul_rn(xk, xl));
    const double p23i = __dadd_rn(__dmul_rn(rk, xl), __dmul_rn(xk, rl));
    return __dsub_rn(__dmul_rn(p01r, p23r), __dmul_rn(p01i, p23i));
}

// Per (snapshot, temperature, pair a < b): the phase overlap
// q_phi = sum_k (re_a re_b + im_a im_b) / sqrt(|a_k|^2 |b_k|^2) / N_eff over
// the sites where both |.|^2 > 1e-24, the Parisi overlap q = sum_k (..) / N
// and, with M quartets, the link overlap q_link = sum_q t_q(a) t_q(b) / M;
// the phase and link overlaps binned on [-1, 1) (bin = (int)((x + 1) / dx),
// clamped), (q, q_link) kept for the scatter at [t][snapshot][pair].
__global__ void deep_pair_kernel(const double* __restrict__ cfg, int N, int NT, int nrep, int nsnap, int nbins,
                                 double dq, const int* __restrict__ quarts, int M,
                                 unsigned long long* __restrict__ phase, unsigned long long* __restrict__ link,
                                 double* __restrict__ scatter) {
    const int npairs = nrep * (nrep - 1) / 2;
    const long long total = (long long)nsnap * NT * npairs;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int pr = (int)(id % npairs);
        const int t = (int)((id / npairs) % NT);
        const long long sn = id / ((long long)npairs * NT);
        int a = 0, rem = pr;
        while (rem >= nrep - 1 - a) { rem -= nrep - 1 - a; a++; }
        const int b = a + 1 + rem;
        const double* x = cfg + ((sn * NT + t) * nrep + a) * 2LL * N;
        const double* y = cfg + ((sn * NT + t) * nrep + b) * 2LL * N;
        double ph = 0.0, rs = 0.0;
        int npm = 0;
        for (int k = 0; k < N; k++) {
            const double ra2 = intensity(x, k), rb2 = intensity(y, k);
            const double dot = __dadd_rn(__dmul_rn(x[2 * k], y[2 * k]), __dmul_rn(x[2 * k + 1], y[2 * k + 1]));
            if (ra2 > 1e-24 && rb2 > 1e-24) {
                ph = __dadd_rn(ph, __ddiv_rn(dot, __dsqrt_rn(__dmul_rn(ra2, rb2))));
                npm++;
            }
        }
        for (int k = 0; k < N; k++)
            rs = __dadd_rn(rs, __dadd_rn(__dmul_rn(x[2 * k], y[2 * k]), __dmul_rn(x[2 * k + 1], y[2 * k + 1])));
        const double qph = npm > 0 ? __ddiv_rn(ph, (double)npm) : 0.0;
        int bin = (int)__ddiv_rn(__dadd_rn(qph, 1.0), dq);
        if (bin < 0) bin = 0;
        if (bin >= nbins) bin = nbins - 1;
        atomicAdd(phase + (size_t)t * nbins + bin, 1ull);
        const double qp = __ddiv_rn(rs, (double)N);
        double ql = 0.0;
        if (M > 0) {
            double ls = 0.0;
            for (int qi = 0; qi < M; qi++)
                ls = __dadd_rn(ls, __dmul_rn(link_term(x, quarts + 5 * qi), link_term(y, quarts + 5 * qi)));
            ql = __ddiv_rn(ls, (double)M);
            int lb = (int)__ddiv_rn(__dadd_rn(ql, 1.0), dq);
            if (lb < 0) lb = 0;
            if (lb >= nbins) lb = nbins - 1;
            atomicAdd(link + (size_t)t * nbins + lb, 1ull);
        }
        double* o = scatter + (((long long)t * nsnap + sn) * npairs + pr) * 2;
        o[0] = qp;
        o[1] = ql;
    }
}

// ---- multi-overlap scatter (analysis_pt.cpp:3468-3643) ----------------------
// On the snapshots snaps[t][0..nit) of each temperature (the reference's
// common iterations, subsampled by its shuffle): meanI[t][r][k] the mean
// intensity over them, summed in that order; then per (t, pair, j) the
// normalised Parisi overlap q = sum re.re+im.im / sqrt(sum I_a sum I_b), the
// phase overlap over sites with both I > 1e-20 (each term divided by
// sqrt(I_a) sqrt(I_b)) and the IFO of I about meanI, as out[t][pair][j][3].
__global__ void multi_mean_kernel(const double* __restrict__ cfg, int N, int NT, int nrep, const int* __restrict__ snaps,
                                  int nit, double* __restrict__ meanI) {
    const long long total = (long long)NT * nrep * N;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(id % N);
        const int r = (int)((id / N) % nrep);
        const int t = (int)(id / ((long long)N * nrep));
        double s = 0.0;
        for (int j = 0; j < nit; j++) {
            const long long sn = snaps[(size_t)t * nit + j];
            s = __dadd_rn(s, intensity(cfg + ((sn * NT + t) * nrep + r) * 2LL * N, k));
        }
        meanI[id] = nit > 0 ? __ddiv_rn(s, (double)nit) : 0.0;
    }
}

__global__ void multi_pair_kernel(const double* __restrict__ cfg, const double* __restrict__ meanI, int N, int NT,
                                  int nrep, const int* __restrict__ snaps, int nit, double* __restrict__ out) {
    const int npairs = nrep * (nrep - 1) / 2;
    const long long total = (long long)NT * npairs * nit;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(id % nit);
        const int pr = (int)((id / nit) % npairs);
        const int t = (int)(id / ((long long)nit * npairs));
        int a = 0, rem = pr;
        while (rem >= nrep - 1 - a) { rem -= nrep - 1 - a; a++; }
        const int b = a + 1 + rem;
        const long long sn = snaps[(size_t)t * nit + j];
        const double* da = cfg + ((sn * NT + t) * nrep + a) * 2LL * N;
        const double* db = cfg + ((sn * NT + t) * nrep + b) * 2LL * N;
        const double* ma_ = meanI + ((size_t)t * nrep + a) * N;
        const double* mb_ = meanI + ((size_t)t * nrep + b) * N;
        double num_q = 0.0, n1q = 0.0, n2q = 0.0, num_qp = 0.0, num_ifo = 0.0, d1 = 0.0, d2 = 0.0;
        int cnt_qp = 0;
        for (int k = 0; k < N; k++) {
            const double Ia = intensity(da, k), Ib = intensity(db, k);
            const double dot = __dadd_rn(__dmul_rn(da[2 * k], db[2 * k]), __dmul_rn(da[2 * k + 1], db[2 * k + 1]));
            num_q = __dadd_rn(num_q, dot);
            n1q = __dadd_rn(n1q, Ia);
            n2q = __dadd_rn(n2q, Ib);
            if (Ia > 1e-20 && Ib > 1e-20) {
                num_qp = __dadd_rn(num_qp, __ddiv_rn(dot, __dmul_rn(__dsqrt_rn(Ia), __dsqrt_rn(Ib))));
                cnt_qp++;
            }
            const double dIa = __dsub_rn(Ia, ma_[k]), dIb = __dsub_rn(Ib, mb_[k]);
            num_ifo = __dadd_rn(num_ifo, __dmul_rn(dIa, dIb));
            d1 = __dadd_rn(d1, __dmul_rn(dIa, dIa));
            d2 = __dadd_rn(d2, __dmul_rn(dIb, dIb));
        }
        const double nrm = __dsqrt_rn(__dmul_rn(n1q, n2q));
        const double den = __dsqrt_rn(__dmul_rn(d1, d2));
        double* o = out + id * 3;
        o[0] = nrm > 0.0 ? __ddiv_rn(num_q, nrm) : 0.0;
        o[1] = cnt_qp > 0 ? __ddiv_rn(num_qp, (double)cnt_qp) : 0.0;
        o[2] = den > 0.0 ? __ddiv_rn(num_ifo, den) : 0.0;
    }
}
}  // namespace pspin

// IFO and experimental-IFO counts of one sample (no reference counterpart as
// a library call): counts [NT][nbins] and valid overlaps [NT] of each; either
// pair of outputs may be NULL.
extern "C" int pspin_ifo_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                     double cmin, double cmax, long long* ifo_counts, long long* ifo_n,
                                     long long* exp_counts, long long* exp_n, const char** err) {
    *err = nullptr;
    if (N < 1 || NT < 1 || nrep < 2 || nsnap < 0 || nbins < 1 || !(cmax > cmin) || !configs ||
        (ifo_counts == nullptr) != (ifo_n == nullptr) || (exp_counts == nullptr) != (exp_n == nullptr)) {
        *err = "pspin_ifo_counts: bad arguments";
        return 1;
    }
    const size_t cnt = (size_t)NT * nbins;
    if (ifo_counts) { memset(ifo_counts, 0, cnt * sizeof(long long)); memset(ifo_n, 0, NT * sizeof(long long)); }
    if (exp_counts) { memset(exp_counts, 0, cnt * sizeof(long long)); memset(exp_n, 0, NT * sizeof(long long)); }
    if (nsnap == 0) return 0;                       // no snapshots: empty histograms
    const size_t n = (size_t)nsnap * NT * nrep * 2 * N;
    const size_t nm = (size_t)NT * nrep * N, nn = (size_t)nsnap * NT * nrep;
    double *d_cfg = nullptr, *d_mean = nullptr, *d_norm = nullptr;
    unsigned long long* d_cnt = nullptr;            // [2][NT][nbins] then [2][NT]
    cudaError_t e = cudaMalloc(&d_cfg, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_mean, nm * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_norm, nn * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, (2 * cnt + 2 * NT) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpy(d_cfg, configs, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, (2 * cnt + 2 * NT) * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        const double dc = (cmax - cmin) / nbins;
        const int threads = 256;
        auto blocks = [&](long long total) { return (int)std::min<long long>((total + threads - 1) / threads, 148LL * 16); };
        const long long npairs = nrep * (nrep - 1) / 2;
        pspin::intensity_mean_kernel<<<blocks((long long)nm), threads>>>(d_cfg, N, NT, nrep, nsnap, d_mean);
        if (ifo_counts) {
            pspin::ifo_norm_kernel<<<blocks((long long)nn), threads>>>(d_cfg, d_mean, N, NT, nrep, nsnap, d_norm);
            pspin::ifo_count_kernel<<<blocks((long long)nsnap * NT * npairs), threads>>>(
                d_cfg, d_mean, d_norm, N, NT, nrep, nsnap, nbins, cmin, dc, d_cnt, d_cnt + 2 * cnt);
        }
        if (exp_counts)
            pspin::exp_ifo_count_kernel<<<blocks((long long)NT * npairs), threads>>>(
                d_mean, N, NT, nrep, nbins, cmin, dc, d_cnt + cnt, d_cnt + 2 * cnt + NT);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> h(2 * cnt + 2 * NT);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d_cnt, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d_cfg);
    cudaFree(d_mean);
    cudaFree(d_norm);
    cudaFree(d_cnt);
    if (e != cudaSuccess) {
        *err = cudaGetErrorString(e);
        return 2;
    }
    for (size_t i = 0; i < cnt; i++) {
        if (ifo_counts) ifo_counts[i] = (long long)h[i];
        if (exp_counts) exp_counts[i] = (long long)h[cnt + i];
    }
    for (int t = 0; t < NT; t++) {
        if (ifo_n) ifo_n[t] = (long long)h[2 * cnt + t];
        if (exp_n) exp_n[t] = (long long)h[2 * cnt + NT + t];
    }
    return 0;
}

// Overlap counts of one sample (no reference counterpart as a library call):
// counts[NT][nbins] over all snapshots and replica pairs of each temperature.
extern "C" int pspin_overlap_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                         double qmin, double qmax, long long* counts, const char** err) {
    *err = nullptr;
    if (N < 1 || NT < 1 || nrep < 2 || nsnap < 0 || nbins < 1 || !(qmax > qmin) || !configs || !counts) {
        *err = "pspin_overlap_counts: bad arguments";
        return 1;
    }
    const size_t n = (size_t)nsnap * NT * nrep * 2 * N;
    double* d_cfg = nullptr;
    unsigned long long* d_cnt = nullptr;
    cudaError_t e = cudaMalloc(&d_cfg, n * sizeof(double) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, (size_t)NT * nbins * sizeof(unsigned long long));
    if (e == cudaSuccess && n) e = cudaMemcpy(d_cfg, configs, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, (size_t)NT * nbins * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        const double dq = (qmax - qmin) / nbins;
        const long long total = (long long)nsnap * NT * (nrep * (nrep - 1) / 2);
        const int threads = 256;
        const int blocks = (int)std::min<long long>((total + threads - 1) / threads, 148LL * 16);
        if (total > 0) pspin::overlap_count_kernel<<<blocks, threads>>>(d_cfg, N, NT, nrep, nsnap, nbins, qmin, dq, d_cnt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(counts, d_cnt, (size_t)NT * nbins * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d_cfg);
    cudaFree(d_cnt);
    if (e != cudaSuccess) {
        *err = cudaGetErrorString(e);
        return 2;
    }
    return 0;
}

// ---- the deeper block and the multi-overlap scatter: host side --------------
static int launch_blocks(long long total) {
    return (int)std::min<long long>((total + 255) / 256, 148LL * 16);
}

// marg [NT][nbins_a2], phase and link [NT][nbins] counts; y
// [nsnap][NT][nrep][3] and scatter [NT][nsnap][npairs][2] values (see the
// kernels).  quartets [M][5] (i, j, k, l, ch) or M = 0: no link overlap.
extern "C" int pspin_deeper_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                        int nbins_a2, double da2, const int32_t* quartets, int M, long long* marg,
                                        double* y, long long* phase, long long* link, double* scatter,
                                        const char** err) {
    *err = nullptr;
    if (N < 1 || NT < 1 || nrep < 2 || nsnap < 0 || nbins < 1 || nbins_a2 < 1 || !(da2 > 0.0) || !configs ||
        M < 0 || (M > 0 && !quartets) || !marg || !y || !phase || !link || !scatter) {
        *err = "pspin_deeper_counts: bad arguments";
        return 1;
    }
    for (int q = 0; q < M; q++)
        for (int c = 0; c < 4; c++)
            if (quartets[5 * q + c] < 0 || quartets[5 * q + c] >= N) {
                *err = "pspin_deeper_counts: quartet site outside [0, N)";
                return 1;
            }
    const long long npairs = (long long)nrep * (nrep - 1) / 2;
    const size_t n = (size_t)nsnap * NT * nrep * 2 * N;
    const size_t nc = (size_t)NT * nbins_a2 + 2 * (size_t)NT * nbins;
    const size_t ny = (size_t)nsnap * NT * nrep * 3, ns = (size_t)NT * nsnap * npairs * 2;
    double *d_cfg = nullptr, *d_y = nullptr, *d_sc = nullptr;
    int* d_q = nullptr;
    unsigned long long* d_cnt = nullptr;
    cudaError_t e = cudaMalloc(&d_cfg, n * sizeof(double) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_y, ny * sizeof(double) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_sc, ns * sizeof(double) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_q, (size_t)5 * M * sizeof(int) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, nc * sizeof(unsigned long long));
    if (e == cudaSuccess && n) e = cudaMemcpy(d_cfg, configs, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && M) e = cudaMemcpy(d_q, quartets, (size_t)5 * M * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, nc * sizeof(unsigned long long));
    if (e == cudaSuccess && nsnap > 0) {
        unsigned long long* d_marg = d_cnt;
        unsigned long long* d_phase = d_cnt + (size_t)NT * nbins_a2;
        unsigned long long* d_link = d_phase + (size_t)NT * nbins;
        pspin::deep_site_kernel<<<launch_blocks((long long)nsnap * NT * nrep), 256>>>(d_cfg, N, NT, nrep, nsnap,
                                                                                      nbins_a2, da2, d_marg, d_y);
        pspin::deep_pair_kernel<<<launch_blocks((long long)nsnap * NT * npairs), 256>>>(
            d_cfg, N, NT, nrep, nsnap, nbins, 2.0 / nbins, d_q, M, d_phase, d_link, d_sc);
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> h(nc);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d_cnt, nc * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && ny) e = cudaMemcpy(y, d_y, ny * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && ns) e = cudaMemcpy(scatter, d_sc, ns * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_cfg);
    cudaFree(d_y);
    cudaFree(d_sc);
    cudaFree(d_q);
    cudaFree(d_cnt);
    if (e != cudaSuccess) {
        *err = cudaGetErrorString(e);
        return 2;
    }
    for (size_t i = 0; i < (size_t)NT * nbins_a2; i++) marg[i] = (long long)h[i];
    for (size_t i = 0; i < (size_t)NT * nbins; i++) {
        phase[i] = (long long)h[(size_t)NT * nbins_a2 + i];
        link[i] = (long long)h[(size_t)NT * nbins_a2 + (size_t)NT * nbins + i];
    }
    return 0;
}

// snaps [NT][nit]: snapshot indices per temperature; out [NT][npairs][nit][3].
extern "C" int pspin_multi_overlap_impl(int N, int NT, int nrep, int nsnap, const double* configs,
                                        const int32_t* snaps, int nit, double* out, const char** err) {
    *err = nullptr;
    if (N < 1 || NT < 1 || nrep < 2 || nsnap < 0 || nit < 0 || !configs || !out || (nit > 0 && !snaps)) {
        *err = "pspin_multi_overlap: bad arguments";
        return 1;
    }
    for (size_t i = 0; i < (size_t)NT * nit; i++)
        if (snaps[i] < 0 || snaps[i] >= nsnap) {
            *err = "pspin_multi_overlap: snapshot index outside [0, nsnap)";
            return 1;
        }
    const long long npairs = (long long)nrep * (nrep - 1) / 2;
    const size_t n = (size_t)nsnap * NT * nrep * 2 * N, no = (size_t)NT * npairs * nit * 3;
    if (no == 0) return 0;
    double *d_cfg = nullptr, *d_mean = nullptr, *d_out = nullptr;
    int* d_s = nullptr;
    cudaError_t e = cudaMalloc(&d_cfg, n * sizeof(double) + 8);
    if (e == cudaSuccess) e = cudaMalloc(&d_mean, (size_t)NT * nrep * N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, no * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_s, (size_t)NT * nit * sizeof(int));
    if (e == cudaSuccess && n) e = cudaMemcpy(d_cfg, configs, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_s, snaps, (size_t)NT * nit * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        pspin::multi_mean_kernel<<<launch_blocks((long long)NT * nrep * N), 256>>>(d_cfg, N, NT, nrep, d_s, nit, d_mean);
        pspin::multi_pair_kernel<<<launch_blocks((long long)NT * npairs * nit), 256>>>(d_cfg, d_mean, N, NT, nrep, d_s,
                                                                                       nit, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, no * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_cfg);
    cudaFree(d_mean);
    cudaFree(d_out);
    cudaFree(d_s);
    if (e != cudaSuccess) {
        *err = cudaGetErrorString(e);
        return 2;
    }
    return 0;
}

// The reference's host sampling, with the same standard-library engines and
// distributions (analysis_pt.cpp:2262-2269, :3504-3507, :3609-3619).
// idx <- 0..n-1 permuted by std::shuffle with std::mt19937(seed): the
// permutation std::shuffle applies to any n-element sequence.
extern "C" int pspin_std_shuffle(int n, uint32_t seed, int32_t* idx) {
    if (n < 0 || (n > 0 && !idx)) return 1;
    for (int i = 0; i < n; i++) idx[i] = i;
    std::mt19937 rng(seed);
    std::shuffle(idx, idx + n, rng);
    return 0;
}

// Reservoir of at most max_pts points (dim doubles each) from a stream of n,
// in stream order, with std::mt19937(seed) and
// std::uniform_int_distribution<int>(0, seen - 1); out [max_pts][dim].
extern "C" int pspin_reservoir_sample(long long n, int dim, const double* pts, int max_pts, uint32_t seed,
                                      double* out, long long* n_out) {
    if (n < 0 || dim < 1 || max_pts < 0 || (n > 0 && !pts) || !out || !n_out) return 1;
    std::mt19937 rng(seed);
    long long kept = 0;
    int total = 0;
    for (long long p = 0; p < n; p++) {
        total++;
        if (kept < max_pts) {
            std::memcpy(out + kept * dim, pts + p * dim, dim * sizeof(double));
            kept++;
        } else {
            std::uniform_int_distribution<int> dist(0, total - 1);
            const int j = dist(rng);
            if (j < max_pts) std::memcpy(out + (long long)j * dim, pts + p * dim, dim * sizeof(double));
        }
    }
    *n_out = kept;
    return 0;
}

// Per block b of counts[b] points (blocks one after another in pts): when a
// block holds more than max_pts, the first max_pts positions of a partial
// Fisher-Yates shuffle (std::uniform_int_distribution<int>(i, size - 1)) with
// one std::mt19937(seed) shared by all blocks in order; out gets each
// block's kept points in order, out_counts their numbers.
extern "C" int pspin_fy_downsample(int nblocks, const long long* counts, int dim, const double* pts, int max_pts,
                                   uint32_t seed, double* out, long long* out_counts) {
    if (nblocks < 0 || dim < 1 || max_pts < 0 || !counts || !out || !out_counts) return 1;
    std::mt19937 rng(seed);
    long long in_off = 0, out_off = 0;
    std::vector<double> pool;
    for (int b = 0; b < nblocks; b++) {
        const long long c = counts[b];
        pool.assign(pts + in_off * dim, pts + (in_off + c) * dim);
        long long keep = c;
        if (c > max_pts) {
            for (int i = 0; i < max_pts; i++) {
                std::uniform_int_distribution<int> dist(i, (int)c - 1);
                const int j = dist(rng);
                for (int d = 0; d < dim; d++) std::swap(pool[(size_t)i * dim + d], pool[(size_t)j * dim + d]);
            }
            keep = max_pts;
        }
        std::memcpy(out + out_off * dim, pool.data(), (size_t)keep * dim * sizeof(double));
        out_counts[b] = keep;
        in_off += c;
        out_off += keep;
    }
    return 0;
}

// Energy decorrelation time tau_E of one temperature's saved energies
// (analysis_pt.cpp:2703-2752): the second half of the M rows [M][nrep],
// replica-averaged, and the first lag whose autocorrelation falls below 1/e,
// interpolated linearly; the reference's loops and operation order.  *tau
// = 0 when the series is too short or has no variance.
extern "C" int pspin_tau_e(int M, int nrep, const double* energy, double* tau) {
    if (M < 0 || nrep < 1 || (M > 0 && !energy) || !tau) return 1;
    *tau = 0.0;
    const int start = M / 2;
    if (start >= M) return 0;
    const int n = M - start;
    if (n < 4) return 0;
    std::vector<double> e_ts(n);
    for (int i = 0; i < n; i++) {
        double sum = 0;
        for (int r = 0; r < nrep; r++) sum += energy[(size_t)(start + i) * nrep + r];
        e_ts[i] = sum / nrep;
    }
    double e_mean = 0, e2_mean = 0;
    for (double v : e_ts) {
        e_mean += v;
        e2_mean += v * v;
    }
    e_mean /= n;
    e2_mean /= n;
    const double var_e = e2_mean - e_mean * e_mean;
    if (var_e <= 0) return 0;
    const double inv_e = 1.0 / 2.7182818284590452354;   // 1/e as the reference computes it (1.0 / M_E)
    double t = 0;
    for (int lag = 1; lag < n / 2; lag++) {
        double c = 0;
        int cnt = 0;
        for (int i = 0; i + lag < n; i++) {
            c += (e_ts[i] - e_mean) * (e_ts[i + lag] - e_mean);
            cnt++;
        }
        c /= cnt;
        const double rho = c / var_e;
        if (rho < inv_e) {
            double c_prev = var_e;
            if (lag > 1) {
                double cp = 0;
                int cnt2 = 0;
                for (int i = 0; i + lag - 1 < n; i++) {
                    cp += (e_ts[i] - e_mean) * (e_ts[i + lag - 1] - e_mean);
                    cnt2++;
                }
                c_prev = cp / cnt2;
            }
            const double rho_prev = c_prev / var_e;
            if (rho_prev > inv_e) t = (lag - 1) + (rho_prev - inv_e) / (rho_prev - rho);
            else t = lag;
            break;
        }
        if (lag == n / 2 - 1) t = lag;
    }
    *tau = t;
    return 0;
}
