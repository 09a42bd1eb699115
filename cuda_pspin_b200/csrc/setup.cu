// setup.cu -- disorder set-up on the device: FMC channel masks, survivor
// counts in quartet-index order, coupling rescale, value gathers from the
// cuRAND stream, and the quartet-index round trip.
//
// Quartet index (test_quartet_index.cu:28-33): for sorted i<j<k<l,
//   q = C(l,4) + C(k,3) + C(j,2) + i.
// The kernels walk q in blocks that share (l,k): block (l,k) covers the
// contiguous range q in [C(l,4)+C(k,3), C(l,4)+C(k,3)+C(k,2)), and inside
// it p = C(j,2)+i.  Blocks in (l,k) lexicographic order are blocks in q
// order, which is what the sparse selection needs (mc_sparse.cu:491-500).
#include "internal.h"
#include <cstdint>

namespace pspin {

__host__ __device__ __forceinline__ int64_t c2(int64_t n) { return n * (n - 1) / 2; }
__host__ __device__ __forceinline__ int64_t c3(int64_t n) { return n * (n - 1) * (n - 2) / 6; }
__host__ __device__ __forceinline__ int64_t c4(int64_t n) { return n * (n - 1) * (n - 2) * (n - 3) / 24; }

// p = C(j,2) + i with i < j -> (i, j)
__device__ __forceinline__ void decode_pair(int64_t p, int& i, int& j) {
    int jj = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while (c2(jj) > p) jj--;
    while (c2(jj + 1) <= p) jj++;
    j = jj;
    i = (int)(p - c2(jj));
}

// disorder.cu:173-180, same operation order: ((w_a + w_b) - w_c) - w_d
__device__ __forceinline__ uint8_t fmc_channel(int i, int j, int k, int l, const double* w, double gamma) {
    const double wi = w[i], wj = w[j], wk = w[k], wl = w[l];
    if (fabs(wi + wj - wk - wl) <= gamma) return 1u;
    if (fabs(wi + wl - wj - wk) <= gamma) return 2u;
    if (fabs(wi + wk - wj - wl) <= gamma) return 4u;
    return 0u;
}

// Channel mask for every q (disorder.cu:153-183).  grid (N, N): block (l, k).
__global__ void fmc_mask_kernel(uint8_t* __restrict__ mask, const double* __restrict__ omega, int N,
                                double gamma) {
    extern __shared__ double w[];
    for (int t = threadIdx.x; t < N; t += blockDim.x) w[t] = omega[t];
    __syncthreads();
    const int l = blockIdx.x, k = blockIdx.y;
    if (l < 3 || k < 2 || k >= l) return;
    const int64_t base = c4(l) + c3(k);
    const int64_t np = c2(k);
    for (int64_t p = threadIdx.x; p < np; p += blockDim.x) {
        int i, j;
        decode_pair(p, i, j);
        mask[base + p] = fmc_channel(i, j, k, l, w, gamma);
    }
}

// Survivor count of block (l, k), written to counts[l*N + k].
__global__ void survivor_count_kernel(unsigned long long* __restrict__ counts, const double* __restrict__ omega,
                                      int N, double gamma) {
    extern __shared__ double w[];
    __shared__ unsigned long long bsum;
    for (int t = threadIdx.x; t < N; t += blockDim.x) w[t] = omega[t];
    if (threadIdx.x == 0) bsum = 0;
    __syncthreads();
    const int l = blockIdx.x, k = blockIdx.y;
    if (l < 3 || k < 2 || k >= l) return;
    const int64_t np = c2(k);
    unsigned int c = 0;
    for (int64_t p = threadIdx.x; p < np; p += blockDim.x) {
        int i, j;
        decode_pair(p, i, j);
        c += __popc(fmc_channel(i, j, k, l, w, gamma));
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&bsum, (unsigned long long)c);
    __syncthreads();
    if (threadIdx.x == 0) counts[(int64_t)l * N + k] = bsum;
}

__global__ void popcount_kernel(const uint8_t* __restrict__ mask, int64_t n, unsigned long long* out) {
    unsigned int c = 0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        c += __popc(mask[q]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

// g4 real parts from the interleaved cuRAND output, scaled and mean-shifted
// (disorder.cu:38-43, 115-124, 200-208: imag dropped, x sigma, +mean on
// non-zero entries)
__global__ void g4_real_kernel(const double* __restrict__ normals, double* __restrict__ g4, int64_t n,
                               double sigma, double mean) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        double v = normals[2 * q] * sigma;
        if (mean != 0.0 && v != 0.0) v += mean;
        g4[q] = v;
    }
}

__global__ void gather_real_kernel(const double* __restrict__ normals, const int64_t* __restrict__ qs, int n,
                                   double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = normals[2 * qs[t]];
}

// test_quartet_index.cu:56-74: decode (the reference's linear scans) ->
// check ordering -> re-encode
__global__ void roundtrip_kernel(int N, int64_t nq, unsigned long long* fails) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int l = 3;
    while (c4(l) <= q) l++;
    l--;
    int64_t rem = q - c4(l);
    int k = 2;
    while (c3(k) <= rem) k++;
    k--;
    rem -= c3(k);
    int j = 1;
    while (c2(j) <= rem) j++;
    j--;
    rem -= c2(j);
    const int i = (int)rem;
    bool bad = (i < 0 || j <= i || k <= j || l <= k || l >= N);
    if (!bad && c4(l) + c3(k) + c2(j) + i != q) bad = true;
    if (bad) atomicAdd(fails, 1ull);
}

// ---------------------------------------------------------------- hosts
cudaError_t dev_fmc_mask(uint8_t* mask, const double* omega, int N, double gamma, cudaStream_t st) {
    fmc_mask_kernel<<<dim3(N, N), 256, N * sizeof(double), st>>>(mask, omega, N, gamma);
    return cudaGetLastError();
}

cudaError_t dev_survivor_counts(unsigned long long* counts, const double* omega, int N, double gamma,
                                cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * (size_t)N * N, st);
    if (e != cudaSuccess) return e;
    survivor_count_kernel<<<dim3(N, N), 256, N * sizeof(double), st>>>(counts, omega, N, gamma);
    return cudaGetLastError();
}

cudaError_t dev_popcount(const uint8_t* mask, int64_t n, unsigned long long* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    popcount_kernel<<<blocks, 256, 0, st>>>(mask, n, out);
    return cudaGetLastError();
}

cudaError_t dev_g4_real(const double* normals, double* g4, int64_t n, double sigma, double mean, cudaStream_t st) {
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    g4_real_kernel<<<blocks, 256, 0, st>>>(normals, g4, n, sigma, mean);
    return cudaGetLastError();
}

cudaError_t dev_gather_real(const double* normals, const int64_t* qs, int n, double* out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    gather_real_kernel<<<(n + 255) / 256, 256, 0, st>>>(normals, qs, n, out);
    return cudaGetLastError();
}

cudaError_t dev_roundtrip(int N, int64_t nq, unsigned long long* fails, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(fails, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (nq <= 0) return cudaSuccess;
    roundtrip_kernel<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(N, nq, fails);
    return cudaGetLastError();
}

}  // namespace pspin
