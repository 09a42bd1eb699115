// pt.cu -- FP64 energies (resync, split) and the device-side replica exchange.
#include "internal.h"
#include "rng.cuh"

namespace pspin {

// ---------------------------------------------------------------------
// FP64 energies of every replica of one unit.
//
// The chain's energy (mc.cu:323-405): E2 = -sum_{i<j} Re[g_ij a_i conj a_j]
// (diagonal excluded), E4 = -sum over active (q,ch) Re[g f_ch(a)] with the
// channel conjugation patterns of mc.cu:389-391.  Amplitudes are the FP32
// ones the sweep evolves, upcast.  With a target, each replica is first
// rescaled in FP64 to sum|a|^2 = target (sphere) or sum|a|^4 = target
// (cube) and the rescaled amplitudes are stored back.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256) energy_kernel(const EnergyParams P) {
    extern __shared__ float2 esm[];
    const Unit U = P.units[blockIdx.x];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N, R = S.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float2* sp = esm;                                                      // [N][32]
    double* red = reinterpret_cast<double*>(esm + (size_t)N * kRepBlock);  // [nw][32][2]
    __shared__ double scale_s[kRepBlock];

    for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
        const int site = idx >> 5, l = idx & 31;
        float2 v = make_float2(0.f, 0.f);
        if (l < U.rep_count) v = P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l];
        sp[idx] = v;
    }
    __syncthreads();

    if (P.target != nullptr) {
        if (warp == 0) {
            double s = 0.0;
            for (int site = 0; site < N; site++) {
                const float2 a = sp[site * kRepBlock + lane];
                const double r2 = (double)a.x * a.x + (double)a.y * a.y;
                s += (S.variant == 0) ? r2 : r2 * r2;
            }
            double sc = 1.0;
            if (lane < U.rep_count && s > 0.0) {
                const double t = P.target[S.rep_off + U.rep_begin + lane];
                sc = (S.variant == 0) ? sqrt(t / s) : sqrt(sqrt(t / s));
            }
            scale_s[lane] = sc;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
            const int site = idx >> 5, l = idx & 31;
            const double sc = scale_s[l];
            const float2 a = sp[idx];
            const float2 b = make_float2((float)(a.x * sc), (float)(a.y * sc));
            sp[idx] = b;
            if (l < U.rep_count) P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l] = b;
        }
        if (P.renorm_only) return;
        __syncthreads();
    }

    double e2 = 0.0, e4 = 0.0;
    if (S.h2_active) {
        const int64_t npair = (int64_t)N * (N - 1) / 2;
        for (int64_t pidx = warp; pidx < npair; pidx += nw) {
            // pair index -> (i<j), row-major over j
            int j = (int)((1.0 + sqrt(1.0 + 8.0 * (double)pidx)) * 0.5);
            while ((int64_t)j * (j - 1) / 2 > pidx) j--;
            while ((int64_t)(j + 1) * j / 2 <= pidx) j++;
            const int i = (int)(pidx - (int64_t)j * (j - 1) / 2);
            const double g = __ldg(P.g2 + S.g2_off + (int64_t)i * N + j);
            if (g == 0.0) continue;
            const float2 ai = sp[i * kRepBlock + lane], aj = sp[j * kRepBlock + lane];
            // -Re[g a_i conj(a_j)]
            e2 -= g * ((double)ai.x * aj.x + (double)ai.y * aj.y);
        }
    }
    const Q64* __restrict__ Q = P.quartets + S.q_off;
    for (int64_t t = warp; t < S.nq; t += nw) {
        const Q64 q = Q[t];
        const int l = q.lch & 0x3FFF, ch = q.lch >> 14;
        const float2 fi = sp[q.i * kRepBlock + lane], fj = sp[q.j * kRepBlock + lane];
        const float2 fk = sp[q.k * kRepBlock + lane], fl = sp[l * kRepBlock + lane];
        double ix = fi.x, iy = fi.y, jx = fj.x, jy = fj.y, kx = fk.x, ky = fk.y, lx = fl.x, ly = fl.y;
        // conjugations: ch0 {k,l}, ch1 {j,k}, ch2 {j,l} (mc.cu:389-391)
        if (ch == 0) { ky = -ky; ly = -ly; }
        else if (ch == 1) { jy = -jy; ky = -ky; }
        else { jy = -jy; ly = -ly; }
        const double ax = ix * jx - iy * jy, ay = ix * jy + iy * jx;   // s0 s1
        const double bx = kx * lx - ky * ly, by = kx * ly + ky * lx;   // s2 s3
        e4 -= q.g * (ax * bx - ay * by);
    }
    red[(warp * kRepBlock + lane) * 2] = e2;
    red[(warp * kRepBlock + lane) * 2 + 1] = e4;
    __syncthreads();
    if (warp == 0 && lane < U.rep_count) {
        double s2 = 0.0, s4 = 0.0;
        for (int w = 0; w < nw; w++) {
            s2 += red[(w * kRepBlock + lane) * 2];
            s4 += red[(w * kRepBlock + lane) * 2 + 1];
        }
        const int64_t gr = S.rep_off + U.rep_begin + lane;
        if (P.e2) P.e2[gr] = s2;
        if (P.e4) P.e4[gr] = s4;
        if (P.energy) {
            if (P.drift) P.drift[gr] = fabs(P.energy[gr] - (s2 + s4));
            P.energy[gr] = s2 + s4;
        }
    }
}

cudaError_t launch_energy(const EnergyParams& p, int n_units, int max_N, cudaStream_t st) {
    if (n_units <= 0) return cudaSuccess;
    const int threads = 256;
    const size_t smem = (size_t)max_N * kRepBlock * sizeof(float2) + (size_t)(threads / 32) * kRepBlock * 2 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(energy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    energy_kernel<<<n_units, threads, smem, st>>>(p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------
// Replica exchange, parallel_tempering.cu:316-352, one thread per sample.
// t runs from the hottest pair upwards and a swap is applied before the
// next t is tried, so a replica may climb several rungs in one pass; the
// uniform is drawn only when delta < 0 (:333-334).  Then betas are
// rebuilt from perm (:347-351).  Thread 0 of block 0 advances the global
// sweep counter.
// ---------------------------------------------------------------------
__global__ void exchange_kernel(const ExchangeParams P) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) *P.sweep_counter += P.nsweeps_done;
    if (!P.do_exchange || s >= P.n_samples) return;
    const SampleDev S = P.samples[s];
    const int NT = P.NT, nr = P.nrep;
    int* perm = P.perm + (int64_t)s * NT * nr;
    const double* E = P.energy + S.rep_off;
    unsigned long long st = P.drand_state[s];
    long long* acc = P.ex_acc + (int64_t)s * (NT - 1);
    long long* prop = P.ex_prop + (int64_t)s * (NT - 1);
    for (int t = 0; t < NT - 1; t++) {
        const double db = P.beta_sched[t] - P.beta_sched[t + 1];
        for (int r = 0; r < nr; r++) {
            const int a = perm[t * nr + r], b = perm[(t + 1) * nr + r];
            const double delta = db * (E[a] - E[b]);
            prop[t]++;
            bool ok = (delta >= 0.0);
            if (!ok) {
                uint64_t st64 = st;
                ok = (drand48_next(st64) < exp(delta));
                st = st64;
            }
            if (ok) {
                acc[t]++;
                perm[t * nr + r] = b;
                perm[(t + 1) * nr + r] = a;
            }
        }
    }
    P.drand_state[s] = st;
    double* beta = P.beta + S.rep_off;
    for (int t = 0; t < NT; t++)
        for (int r = 0; r < nr; r++) beta[perm[t * nr + r]] = P.beta_sched[t];
}

cudaError_t launch_exchange(const ExchangeParams& p, cudaStream_t st) {
    const int threads = 128;
    const int blocks = p.n_samples > 0 ? (p.n_samples + threads - 1) / threads : 1;
    exchange_kernel<<<blocks, threads, 0, st>>>(p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------
// Observable series: one warp per sample.  E of the nrep replicas at the
// slot and q_ab = Re sum_k a_k^a conj(a_k^b) / N for every pair a < b
// (the overlap of analysis_pt.cpp:1404-1416), summed in FP64.
// ---------------------------------------------------------------------
__global__ void observe_kernel(const ObserveParams P) {
    const int s = blockIdx.x, lane = threadIdx.x;
    const long long row = (*P.sweep_counter - P.sweep0) / P.pt_freq - 1;
    if (s >= P.n_samples || row < 0 || row >= P.capacity) return;
    const SampleDev S = P.samples[s];
    const int nr = P.nrep;
    const int npairs = nr * (nr - 1) / 2;
    const int* perm = P.perm + ((int64_t)s * P.NT + P.temp_index) * nr;
    const int64_t base = row * P.n_samples + s;
    for (int r = lane; r < nr; r += 32) P.E_out[base * nr + r] = P.energy[S.rep_off + perm[r]];
    int pr = 0;
    for (int a = 0; a < nr; a++)
        for (int b = a + 1; b < nr; b++, pr++) {
            const float2* xa = P.spins + S.spin_off + perm[a];
            const float2* xb = P.spins + S.spin_off + perm[b];
            double acc = 0.0;
            for (int k = lane; k < S.N; k += 32) {
                const float2 u = xa[(int64_t)k * S.R], v = xb[(int64_t)k * S.R];
                acc += (double)u.x * v.x + (double)u.y * v.y;
            }
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
            if (lane == 0) P.q_out[base * npairs + pr] = acc / S.N;
        }
}

cudaError_t launch_observe(const ObserveParams& p, cudaStream_t st) {
    if (p.n_samples <= 0) return cudaSuccess;
    observe_kernel<<<p.n_samples, 32, 0, st>>>(p);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------
// FP32 FMA throughput probe: 8 independent register chains per thread, so
// the FMA pipe, not latency, is the limit.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters) {
    float a[8];
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = (float)(threadIdx.x + c) * 1e-3f;
    const float m = 0.999999f, k = 1e-7f;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < 8; c++) a[c] = fmaf(a[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) s += a[c];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// the same with paired FMA (fma.rn.f32x2): 8 chains of two lanes each
__global__ void __launch_bounds__(256) fma2_probe_kernel(float* out, int iters) {
    float2 a[8];
#pragma unroll
    for (int c = 0; c < 8; c++) a[c] = make_float2((float)(threadIdx.x + c) * 1e-3f, (float)(threadIdx.x - c) * 1e-3f);
    const float2 m = make_float2(0.999999f, 0.999998f), k = make_float2(1e-7f, 2e-7f);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < 8; c++) a[c] = __ffma2_rn(a[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) s += a[c].x + a[c].y;
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// paired = 1: the fma.rn.f32x2 probe (twice the FMA per thread and iteration)
cudaError_t launch_fma_probe(float* out, int blocks, int iters, cudaStream_t st, int paired) {
    if (paired) fma2_probe_kernel<<<blocks, 256, 0, st>>>(out, iters);
    else fma_probe_kernel<<<blocks, 256, 0, st>>>(out, iters);
    return cudaGetLastError();
}

}  // namespace pspin
