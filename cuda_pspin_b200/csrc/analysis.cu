// analysis.cu -- overlap histograms of saved configurations on the GPU: the
// hot loops of the reference's analysis_pt.cpp for the Parisi P(q)
// (:1337-1437), the intensity fluctuation overlap IFO (:1498-1619) and the
// experimental IFO of time-averaged spectra (:1679-1806).
//
// configs: [nsnap][NT][nrep][N][2] doubles (the body of configs.bin without
// the per-snapshot sweep numbers).  One thread per (snapshot, temperature,
// replica pair a < b): q = Re sum_k a_k conj(b_k) / N summed over k in order
// with round-to-nearest products and sums, no contraction, like the
// reference's loop, so every q falls in the same bin:
// bin = (int)((q - qmin) / dq), clamped to [0, nbins).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
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
