// tcfield.cu -- all-site local fields of every replica as a tensor-core
// contraction with split-BF16 operands (tcgen05, FP32 accumulation in TMEM),
// and the FP64 all-site fields it is checked against.
//
// Pair space.  For pairs P = (u1<u2) let A_P = a_u1 a_u2.  A quartet in
// channel ch has an unconjugated pair U and a conjugated pair C
// (disorder.h:9-16), so H4 = -Re sum_{P,Q} W[P,Q] A_P conj(A_Q) with
// W[U,C] = g.  With the symmetric Ws = W + W^T,
//     F = Ws conj(A)                       (one real GEMM per re/im column)
//     h_m = sum_{p != m} a_p F_(m,p) + sum_{j != m} g2_mj conj(a_j)
//     E4  = -1/2 Re sum_P A_P F_P ,
// h_m being the field of site m (dE of a one-site change = -Re[da_m h_m]).
//
// Split BF16 (Henry, Tang & Heinecke, "Leveraging the bfloat16 AI datatype
// for higher-precision computations", ARITH 2019): x = hi + lo with
// hi = bf16(x), lo = bf16(x - hi); Ws X ~ Ws_hi X_hi + Ws_hi X_lo + Ws_lo X_hi.
// The three products are one GEMM over a concatenated K:
//     [Ws_hi | Ws_hi | Ws_lo] (M x 3K)  x  [X_hi ; X_lo ; X_hi] (3K x 2R),
// accumulated in FP32 by the sm100 UMMA pipeline (CUTLASS 4.5 collective:
// TMA loads, tcgen05.mma, TMEM accumulator).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "cute/tensor.hpp"
#include "cutlass/cutlass.h"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/gemm/collective/collective_builder.hpp"
#include "cutlass/gemm/device/gemm_universal_adapter.h"
#include "cutlass/gemm/kernel/gemm_universal.hpp"
#include "cutlass/util/packed_stride.hpp"

#include "internal.h"

namespace pspin {

namespace tc {
using namespace cute;
using ElementA = cutlass::bfloat16_t;
using ElementB = cutlass::bfloat16_t;
using ElementC = float;
using ElementAcc = float;
using LayoutA = cutlass::layout::RowMajor;      // Ws' [M][3K]   (K-major)
using LayoutB = cutlass::layout::ColumnMajor;   // X'  [2R][3K]  (K-major)
using LayoutC = cutlass::layout::RowMajor;      // F   [M][2R]
using MmaTileShape = Shape<_128, _128, _64>;
using ClusterShape = Shape<_1, _1, _1>;
using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, MmaTileShape, ClusterShape,
    cutlass::epilogue::collective::EpilogueTileAuto, ElementAcc, ElementAcc, ElementC, LayoutC, 4, ElementC,
    LayoutC, 4, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;
using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementA, LayoutA, 8, ElementB, LayoutB, 8, ElementAcc,
    MmaTileShape, ClusterShape,
    cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
    cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;
using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, void>;
using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;
}  // namespace tc

// F[M][NC] = Ws'[M][K3] x X'^T, X' stored [NC][K3]
cudaError_t tc_gemm(int M, int NC, int K3, const __nv_bfloat16* A, const __nv_bfloat16* B, float* F, void* workspace,
                    size_t ws_bytes, cudaStream_t st, size_t* ws_needed) {
    using namespace tc;
    using StrideA = typename Gemm::GemmKernel::StrideA;
    using StrideB = typename Gemm::GemmKernel::StrideB;
    using StrideC = typename Gemm::GemmKernel::StrideC;
    using StrideD = typename Gemm::GemmKernel::StrideD;
    StrideA sA = cutlass::make_cute_packed_stride(StrideA{}, {M, K3, 1});
    StrideB sB = cutlass::make_cute_packed_stride(StrideB{}, {NC, K3, 1});
    StrideC sC = cutlass::make_cute_packed_stride(StrideC{}, {M, NC, 1});
    StrideD sD = cutlass::make_cute_packed_stride(StrideD{}, {M, NC, 1});
    typename Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,
                                  {M, NC, K3, 1},
                                  {reinterpret_cast<const ElementA*>(A), sA, reinterpret_cast<const ElementB*>(B), sB},
                                  {{1.0f, 0.0f}, F, sC, F, sD}};
    Gemm g;
    if (ws_needed) {
        *ws_needed = Gemm::get_workspace_size(args);
        return cudaSuccess;
    }
    if (g.can_implement(args) != cutlass::Status::kSuccess) return cudaErrorInvalidValue;
    if (g.initialize(args, workspace, st) != cutlass::Status::kSuccess) return cudaErrorInvalidValue;
    if (g.run(st) != cutlass::Status::kSuccess) return cudaErrorLaunchFailure;
    return cudaGetLastError();
}

__device__ __forceinline__ int pair_index(int u1, int u2) { return u2 * (u2 - 1) / 2 + u1; }  // u1 < u2

// Ws (FP32, [M][Kp], zero padded) -> [Ws_hi | Ws_hi | Ws_lo] as BF16 [M][3Kp]
__global__ void split_ws_kernel(const float* __restrict__ ws, __nv_bfloat16* __restrict__ out, int M, int Kp) {
    const int64_t n = (int64_t)M * Kp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / Kp, col = t % Kp;
        const float x = ws[t];
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
        __nv_bfloat16* o = out + row * 3 * Kp;
        o[col] = hi;
        o[Kp + col] = hi;
        o[2 * Kp + col] = lo;
    }
}

// X' [2R][3Kp]: column 2r = Re conj(A_P), 2r+1 = Im conj(A_P), split as
// [X_hi ; X_lo ; X_hi] along K
__global__ void pair_split_kernel(const float2* __restrict__ spins, int N, int R, int npairs, int Kp,
                                  __nv_bfloat16* __restrict__ X) {
    const int r = blockIdx.y;
    for (int P = blockIdx.x * blockDim.x + threadIdx.x; P < Kp; P += gridDim.x * blockDim.x) {
        float re = 0.f, im = 0.f;
        if (P < npairs) {
            int u2 = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)P)) * 0.5f);
            while (u2 * (u2 - 1) / 2 > P) u2--;
            while ((u2 + 1) * u2 / 2 <= P) u2++;
            const int u1 = P - u2 * (u2 - 1) / 2;
            const float2 a = spins[(int64_t)u1 * R + r], b = spins[(int64_t)u2 * R + r];
            re = a.x * b.x - a.y * b.y;          // A_P = a_u1 a_u2
            im = -(a.x * b.y + a.y * b.x);       // conjugated
        }
        const float v[2] = {re, im};
        for (int c = 0; c < 2; c++) {
            const __nv_bfloat16 hi = __float2bfloat16_rn(v[c]);
            const __nv_bfloat16 lo = __float2bfloat16_rn(v[c] - __bfloat162float(hi));
            __nv_bfloat16* o = X + (int64_t)(2 * r + c) * 3 * Kp;
            o[P] = hi;
            o[Kp + P] = lo;
            o[2 * Kp + P] = hi;
        }
    }
}

// h_m = sum_p a_p F_(m,p) + sum_j g2_mj conj(a_j);  E4 = -1/2 Re sum_P A_P F_P,
// E2 = -1/2 Re sum_m a_m h2_m.  One block per replica.
__global__ void site_fields_kernel(const float2* __restrict__ spins, int N, int R, const float* __restrict__ F,
                                   int NC, const double* __restrict__ g2, int h2_active, float2* __restrict__ h,
                                   double* __restrict__ e2, double* __restrict__ e4) {
    const int r = blockIdx.x;
    double s2 = 0.0, s4 = 0.0;
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        const float2 am = spins[(int64_t)m * R + r];
        float hx = 0.f, hy = 0.f, gx = 0.f, gy = 0.f;
        for (int p = 0; p < N; p++) {
            if (p == m) continue;
            const float2 ap = spins[(int64_t)p * R + r];
            const int P = m < p ? pair_index(m, p) : pair_index(p, m);
            const float fx = F[(int64_t)P * NC + 2 * r], fy = F[(int64_t)P * NC + 2 * r + 1];
            hx += ap.x * fx - ap.y * fy;
            hy += ap.x * fy + ap.y * fx;
            if (p > m) s4 += (double)((am.x * ap.x - am.y * ap.y) * fx - (am.x * ap.y + am.y * ap.x) * fy);
            if (h2_active) {
                const float g = (float)g2[(int64_t)m * N + p];
                gx += g * ap.x;
                gy -= g * ap.y;
            }
        }
        s2 += (double)(am.x * gx - am.y * gy);
        h[(int64_t)r * N + m] = make_float2(hx + gx, hy + gy);
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = s2;
    red[1][threadIdx.x] = s4;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int t = 0; t < (int)blockDim.x; t++) { a += red[0][t]; b += red[1][t]; }
        e2[r] = -0.5 * a;
        e4[r] = -0.5 * b;
    }
}

// FP64 all-site fields from the quartet table (the oracle form, upcast
// amplitudes); one block per replica, lanes over the table.
__global__ void fp64_fields_kernel(const float2* __restrict__ spins, int N, int R, const Q64* __restrict__ Q,
                                   int64_t nq, const double* __restrict__ g2, int h2_active,
                                   double2* __restrict__ h) {
    extern __shared__ double2 hs[];
    const int r = blockIdx.x;
    for (int m = threadIdx.x; m < N; m += blockDim.x) hs[m] = make_double2(0.0, 0.0);
    __syncthreads();
    static const int U[3][2] = {{0, 1}, {0, 3}, {0, 2}};
    for (int64_t t = threadIdx.x; t < nq; t += blockDim.x) {
        const Q64 q = Q[t];
        const int ch = q.lch >> 14;
        const int s[4] = {q.i, q.j, q.k, q.lch & 0x3FFF};
        double2 a[4];
        for (int k = 0; k < 4; k++) {
            const float2 v = spins[(int64_t)s[k] * R + r];
            a[k] = make_double2(v.x, v.y);
        }
        const int u0 = U[ch][0], u1 = U[ch][1];
        int c0 = -1, c1 = -1;
        for (int k = 0; k < 4; k++)
            if (k != u0 && k != u1) { if (c0 < 0) c0 = k; else c1 = k; }
        // member k: partner p, opposite o1, o2 -> g a_p conj(a_o1) conj(a_o2)
        for (int k = 0; k < 4; k++) {
            int p, o1, o2;
            if (k == u0) { p = u1; o1 = c0; o2 = c1; }
            else if (k == u1) { p = u0; o1 = c0; o2 = c1; }
            else if (k == c0) { p = c1; o1 = u0; o2 = u1; }
            else { p = c0; o1 = u0; o2 = u1; }
            const double ox = a[o1].x * a[o2].x - a[o1].y * a[o2].y;
            const double oy = -(a[o1].x * a[o2].y + a[o1].y * a[o2].x);   // conj(a_o1 a_o2)
            const double vx = q.g * (a[p].x * ox - a[p].y * oy);
            const double vy = q.g * (a[p].x * oy + a[p].y * ox);
            atomicAdd(&hs[s[k]].x, vx);
            atomicAdd(&hs[s[k]].y, vy);
        }
    }
    __syncthreads();
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double hx = hs[m].x, hy = hs[m].y;
        if (h2_active)
            for (int j = 0; j < N; j++) {
                if (j == m) continue;
                const float2 v = spins[(int64_t)j * R + r];
                const double g = g2[(int64_t)m * N + j];
                hx += g * v.x;
                hy -= g * v.y;
            }
        h[(int64_t)r * N + m] = make_double2(hx, hy);
    }
}

cudaError_t launch_split_ws(const float* ws, __nv_bfloat16* out, int M, int Kp, cudaStream_t st) {
    split_ws_kernel<<<148 * 8, 256, 0, st>>>(ws, out, M, Kp);
    return cudaGetLastError();
}

cudaError_t launch_pair_split(const float2* spins, int N, int R, int npairs, int Kp, __nv_bfloat16* X,
                              cudaStream_t st) {
    dim3 grid((Kp + 255) / 256, R);
    pair_split_kernel<<<grid, 256, 0, st>>>(spins, N, R, npairs, Kp, X);
    return cudaGetLastError();
}

cudaError_t launch_site_fields(const float2* spins, int N, int R, const float* F, int NC, const double* g2,
                               int h2_active, float2* h, double* e2, double* e4, cudaStream_t st) {
    site_fields_kernel<<<R, 256, 0, st>>>(spins, N, R, F, NC, g2, h2_active, h, e2, e4);
    return cudaGetLastError();
}

cudaError_t launch_fp64_fields(const float2* spins, int N, int R, const Q64* Q, int64_t nq, const double* g2,
                               int h2_active, double2* h, cudaStream_t st) {
    fp64_fields_kernel<<<R, 256, N * sizeof(double2), st>>>(spins, N, R, Q, nq, g2, h2_active, h);
    return cudaGetLastError();
}

}  // namespace pspin
