// noalloc.cu -- FMC survivor counting that allocates nothing.
//
// Some callers cannot call cudaMalloc: host frameworks that own every
// device allocation through their own pool (a second allocator would
// fragment or overcommit the memory the pool has reserved), and plugins
// that only receive device pointers from their host and may not take
// device memory of their own.  pspin_fmc_survivors_static counts the
// quartet-channel pairs that survive the frequency-matching filter (the
// count the sparse set-up draws its quartets from) with its intermediate
// per-row counts in a file-scope device array instead of a cudaMalloc'd
// buffer.  The caller passes the frequencies and the output as device
// pointers.
//
// Limits and sharing:
//  * N <= kStaticMaxN (1024); larger N is rejected with PSPIN_ERR_ARG.
//  * The array (3 * 1024 counters, 24 KB) lives in every GPU that loads
//    libpspin.so until the process exits.
//  * All calls share the one array and it keeps the last call's contents.
//    Each call overwrites every row it reads, so nothing has to start at
//    zero, but calls that overlap on the GPU (different streams, or
//    different host threads on one device) race on it.
//  * The device address of the array is looked up with
//    cudaGetSymbolAddress by the first call on each device (with that
//    device current) and kept for that device's CUDA context; a call in a
//    new context (after cudaDeviceReset, say) looks it up again.  Make the
//    first call on a device before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/pspin.h"

namespace pspin {

constexpr int kStaticMaxN = 1024;
constexpr int kMaxDevices = 64;

// per-l survivor counts of the three channels
static __device__ __align__(256) unsigned long long g_survivor_rows[kStaticMaxN * 3];

__device__ __forceinline__ long long c2s(long long n) { return n * (n - 1) / 2; }

// Block l counts every quartet i<j<k<l of the channel it passes first
// (disorder.cu:173-180, same operation order) and writes row l.
__global__ void survivor_rows_kernel(unsigned long long* rows, const double* __restrict__ omega, int N,
                                     double gamma) {
    __shared__ double w[kStaticMaxN];
    __shared__ unsigned long long part[3][8];
    for (int t = threadIdx.x; t < N; t += blockDim.x) w[t] = omega[t];
    __syncthreads();
    const int l = blockIdx.x;
    unsigned int c0 = 0, c1 = 0, c2 = 0;
    if (l >= 3) {
        const double wl = w[l];
        for (int k = 2; k < l; k++) {
            const double wk = w[k];
            const long long np = c2s(k);
            for (long long p = threadIdx.x; p < np; p += blockDim.x) {
                int j = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
                while (c2s(j) > p) j--;
                while (c2s(j + 1) <= p) j++;
                const int i = (int)(p - c2s(j));
                const double wi = w[i], wj = w[j];
                if (fabs(wi + wj - wk - wl) <= gamma) c0++;
                else if (fabs(wi + wl - wj - wk) <= gamma) c1++;
                else if (fabs(wi + wk - wj - wl) <= gamma) c2++;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_down_sync(0xffffffffu, c0, o);
        c1 += __shfl_down_sync(0xffffffffu, c1, o);
        c2 += __shfl_down_sync(0xffffffffu, c2, o);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { part[0][warp] = c0; part[1][warp] = c1; part[2][warp] = c2; }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += part[threadIdx.x][q];
        rows[(size_t)l * 3 + threadIdx.x] = s;
    }
}

// out[0] = total, out[1..3] = channels 0..2, summed over rows 0..N-1
__global__ void survivor_sum_kernel(const unsigned long long* rows, int N, int64_t* out) {
    unsigned long long s0 = 0, s1 = 0, s2 = 0;
    for (int l = threadIdx.x; l < N; l += 32) {
        s0 += rows[(size_t)l * 3];
        s1 += rows[(size_t)l * 3 + 1];
        s2 += rows[(size_t)l * 3 + 2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if (threadIdx.x == 0) {
        out[0] = (int64_t)(s0 + s1 + s2);
        out[1] = (int64_t)s0;
        out[2] = (int64_t)s1;
        out[3] = (int64_t)s2;
    }
}

static std::mutex g_addr_mu;
static unsigned long long* g_addr[kMaxDevices] = {};
static unsigned long long g_ctx_id[kMaxDevices] = {};   // context the cached address belongs to

// Unique id of the calling thread's current CUDA context (ids are never
// reused within a process), through driver entry points the runtime hands
// out; 0 when there is no current context or the entry points are missing.
static unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
        cudaGetLastError();
    }
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx) return 0;
    if (get_id(ctx, &id) != 0) return 0;
    return id;
}

}  // namespace pspin

namespace pspin {
int report_error(int code, const std::string& msg);   // abi.cu: sets pspin_last_error()
}

using namespace pspin;

extern "C" int pspin_fmc_survivors_static(int N, const double* d_omega, double gamma, int64_t* d_counts,
                                          void* stream) {
    if (N < 4 || N > kStaticMaxN) {
        return report_error(PSPIN_ERR_ARG, "pspin_fmc_survivors_static: N=" + std::to_string(N) +
                                               " outside [4, " + std::to_string(kStaticMaxN) +
                                               "], the size of its static scratch array");
    }
    if (!d_omega || !d_counts) {
        return report_error(PSPIN_ERR_ARG, "pspin_fmc_survivors_static: null device pointer");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        return report_error(PSPIN_ERR_CUDA,
                            std::string("pspin_fmc_survivors_static: no current device: ") + cudaGetErrorString(e));
    }
    unsigned long long* rows = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_addr_mu);
        const unsigned long long ctx = current_context_id();
        if (!g_addr[dev] || ctx == 0 || ctx != g_ctx_id[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_survivor_rows);
            if (e != cudaSuccess || !p) {
                g_addr[dev] = nullptr;
                return report_error(PSPIN_ERR_CUDA,
                                    std::string("pspin_fmc_survivors_static: cudaGetSymbolAddress failed: ") +
                                        cudaGetErrorString(e));
            }
            g_addr[dev] = static_cast<unsigned long long*>(p);
            g_ctx_id[dev] = current_context_id();   // the look-up made the context current if it was not
        }
        rows = g_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    survivor_rows_kernel<<<N, 256, 0, st>>>(rows, d_omega, N, gamma);
    survivor_sum_kernel<<<1, 32, 0, st>>>(rows, N, d_counts);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        return report_error(PSPIN_ERR_CUDA,
                            std::string("pspin_fmc_survivors_static: launch failed: ") + cudaGetErrorString(e));
    }
    return PSPIN_OK;
}
