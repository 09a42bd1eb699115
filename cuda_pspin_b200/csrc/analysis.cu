// analysis.cu -- overlap histograms of saved configurations on the GPU (the
// hot loop of the reference's analysis_pt.cpp:1337-1437, Parisi P(q)).
//
// configs: [nsnap][NT][nrep][N][2] doubles (the body of configs.bin without
// the per-snapshot sweep numbers).  One thread per (snapshot, temperature,
// replica pair a < b): q = Re sum_k a_k conj(b_k) / N summed over k in order
// with round-to-nearest products and sums, no contraction, like the
// reference's loop, so every q falls in the same bin:
// bin = (int)((q - qmin) / dq), clamped to [0, nbins).
#include <cuda_runtime.h>
#include <cstdint>
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

}  // namespace pspin

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
