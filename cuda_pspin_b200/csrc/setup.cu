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
#include <algorithm>
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

// ---- g2 (disorder.cu:45-80, 130-143, 191-197; mc.cu:469-477, 436-502) ------
// g2[i][j] <- Re of normal (min(i,j), max(i,j)) (imaginary parts dropped,
// lower triangle copied from the upper one, diagonal kept); with uniform
// FMC, i != j with |w_i - w_j| > gamma set to 0 (both halves); *count <- the
// non-zero entries with i <= j.
__global__ void g2_build_kernel(const double* __restrict__ normals, int N, const double* __restrict__ omega,
                                double gamma, double* __restrict__ g2, unsigned long long* __restrict__ count) {
    const long long total = (long long)N * N;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(id / N), j = (int)(id % N);
        const long long src = (i > j) ? (long long)j * N + i : (long long)i * N + j;
        double v = normals[2 * src];
        if (omega != nullptr && i != j && fabs(omega[i] - omega[j]) > gamma) v = 0.0;
        g2[id] = v;
        if (i <= j && v != 0.0) atomicAdd(count, 1ull);
    }
}

// g2 <- g2 sigma, then + mean on the non-zero entries
__global__ void g2_scale_kernel(double* __restrict__ g2, long long n, double sigma, double mean, int shift) {
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n;
         id += (long long)gridDim.x * blockDim.x) {
        double v = g2[id] * sigma;
        if (shift && v != 0.0) v += mean;
        g2[id] = v;
    }
}

// ---- replica initialisation (spins.cu:27-69, 84-111; spins_sparse.cu:28-80)
// One CTA per replica, blockDim as the reference launches its normalisation
// (sphere: N up to 1024, cube: N rounded up to a multiple of 32, >= 32, up to
// 1024), the same shared-memory tree and expressions, so the scale is the
// reference's -- including its truncation for N not a power of two (the
// tree starts at blockDim/2) and, for the cube beyond 1024 sites, scaling
// only the first 1024.  exact = 1 (or a sphere beyond 1024 sites, which the
// reference sums on the host) sums every site in order instead.  The
// amplitudes are written as FP32 into the sample's [site][replica] layout,
// target[r] <- the constraint value of the scaled amplitudes (FP64, in site
// order).
__global__ void normalize_replicas_kernel(const double* __restrict__ nrm, int N, int R, int cube, int exact,
                                          float2* __restrict__ spins, double* __restrict__ target) {
    extern __shared__ double sdata[];
    const int r = blockIdx.x, tid = threadIdx.x;
    const double* a = nrm + (size_t)r * 2 * N;
    __shared__ double scale_s;
    const bool seq = exact || (!cube && N > 1024);
    if (seq) {
        if (tid == 0) {
            double sum = 0.0;
            for (int i = 0; i < N; i++) {
                const double r2 = __dadd_rn(__dmul_rn(a[2 * i], a[2 * i]), __dmul_rn(a[2 * i + 1], a[2 * i + 1]));
                sum = __dadd_rn(sum, cube ? __dmul_rn(r2, r2) : r2);
            }
            scale_s = cube ? pow((double)N / sum, 0.25) : sqrt((double)N / sum);
        }
    } else {
        double local = 0.0;
        if (tid < N) {
            const double re = a[2 * tid], im = a[2 * tid + 1];
            if (cube) {
                const double r2 = re * re + im * im;
                local = r2 * r2;
            } else {
                local = re * re + im * im;
            }
        }
        sdata[tid] = local;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (tid < s) sdata[tid] += sdata[tid + s];
            __syncthreads();
        }
        if (tid == 0) scale_s = cube ? pow((double)N / sdata[0], 0.25) : sqrt((double)N / sdata[0]);
    }
    __syncthreads();
    const double scale = scale_s;
    const int lim = (seq || !cube) ? N : min(N, (int)blockDim.x);
    for (int i = tid; i < N; i += blockDim.x) {
        double re = a[2 * i], im = a[2 * i + 1];
        if (i < lim) {
            re *= scale;
            im *= scale;
        }
        spins[(size_t)i * R + r] = make_float2((float)re, (float)im);
    }
    if (tid == 0) {
        double t = 0.0;
        for (int i = 0; i < N; i++) {
            double re = a[2 * i], im = a[2 * i + 1];
            if (i < lim) {
                re = __dmul_rn(re, scale);
                im = __dmul_rn(im, scale);
            }
            const double r2 = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
            t = __dadd_rn(t, cube ? __dmul_rn(r2, r2) : r2);
        }
        target[r] = t;
    }
}

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


cudaError_t dev_g2_build(const double* normals, int N, const double* omega, double gamma, double* g2,
                         unsigned long long* count, cudaStream_t st) {
    const long long total = (long long)N * N;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
    g2_build_kernel<<<blocks, 256, 0, st>>>(normals, N, omega, gamma, g2, count);
    return cudaGetLastError();
}

cudaError_t dev_g2_scale(double* g2, long long n, double sigma, double mean, int shift, cudaStream_t st) {
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    if (n > 0) g2_scale_kernel<<<blocks, 256, 0, st>>>(g2, n, sigma, mean, shift);
    return cudaGetLastError();
}

// the reference's block size for each normalisation (spins.cu:89, spins_sparse.cu:76)
cudaError_t dev_normalize_replicas(const double* nrm, int N, int R, int cube, int exact, float2* spins,
                                   double* target, cudaStream_t st) {
    int bd = (N < 1024) ? N : 1024;
    if (cube) {
        bd = (N < 1024) ? (N + 31) / 32 * 32 : 1024;
        if (bd < 32) bd = 32;
    }
    if (R > 0)
        normalize_replicas_kernel<<<R, bd, bd * sizeof(double), st>>>(nrm, N, R, cube, exact, spins, target);
    return cudaGetLastError();
}

}  // namespace pspin
