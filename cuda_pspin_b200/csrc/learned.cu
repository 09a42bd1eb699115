// learned.cu -- the sweep with local fields at both ends of every move, used
// (mode 1) to record accepted plain moves for training and (mode 2) to run
// the learned proposal with the exact Metropolis-Hastings correction; and
// the network's training kernels (forward, backward, Adam).
//
// Two field passes per move.  Pass 1 reads site i's and site j's lists at
// the current state x: h_i(x), h_j(x) (the proposal's features).  Pass 2
// reads only the pair's sub-lists (the terms of h_i that contain a_j and of
// h_j that contain a_i, about 3/N of a site list) with the changes da_i,
// da_j in the pair's slots, giving h_i(x') - h_i(x) and h_j(x') - h_j(x)
// (the reverse density's features).  E is affine in each site, so
//     dE = -Re[da_i h_i(x')] - Re[da_j h_j(x)]
// exactly (h_i(x') is h_i with a_j' in place, h_j(x) is h_j with a_i).
#include <cuda_bf16.h>

#include "../../include/pspin.h"
#include "mlp.cuh"
#include "sweep_common.cuh"

namespace pspin {

struct LearnParams {
    int mode;                       // 1: plain proposal, fields + recording; 2: learned proposal
    const __nv_bfloat16* w;         // network weights [kMlpParams]
    float* records;                 // ring of accepted plain moves [cap][kRecordFloats]
    unsigned long long* rec_count;  // moves written so far (ring position = count % cap)
    int rec_cap;
    float rec_prob;
};

// Network evaluation for the CTA's 32 replicas by all its warps, on the
// tensor cores with warp-level mma.sync m16n8k16 (BF16 operands, FP32
// accumulation): each layer is Out[32 x units] = In[32 x K] W^T, two m16
// tiles of replicas x n8 tiles of units, the n8 tiles spread over the warps.
// A fragments come from the activations in shared memory, stored already
// rounded to BF16 with two consecutive inputs of one replica in one 32-bit
// word (row kp holds inputs 2kp, 2kp+1 of the 32 replicas; row stride
// kActStride = 40 words, so the 8 row groups x 4 column pairs of a fragment
// load hit 32 distinct banks).  B fragments come straight from the BF16
// weight rows in global memory (12.9 KB, L1-resident; two consecutive
// inputs of one unit are one 32-bit word).  Bias and tanh in the FP32
// epilogue, which packs the lane's two units back into one word.  K is
// padded to 16 (first layer) and the 26 outputs to 32 with zeros; the
// outputs stay FP32 (row stride kOutStride).  (32 x 64 tiles are below
// tcgen05's smallest M of 64, and the step is latency-bound.)  Fragment
// layouts: PTX ISA, "Matrix Fragments for mma.m16n8k16 with floating point
// type".
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

constexpr int kActStride = 40;    // words per packed activation row (32 replicas + 8 pad)
constexpr int kOutStride = 36;    // floats per output row (32 replicas + 4 pad)

// One layer: X [ceil(K/2)][kActStride] packed BF16 pairs in shared memory ->
// Y, packed the same way (HIDDEN: tanh) or FP32 [units][kOutStride] (the
// output layer); weights w[u*K + k] (BF16, global), bias bias[u]
template <int K, int UNITS, bool HIDDEN>
__device__ __forceinline__ void mlp_layer_mma(const __nv_bfloat16* __restrict__ w, const __nv_bfloat16* __restrict__ bias,
                                              const uint32_t* X, void* Y, int warp, int W, int lane) {
    constexpr int KP = K < 16 ? 16 : K;          // padded K
    constexpr int NT = (UNITS + 7) / 8;          // n8 tiles
    const int g = lane >> 2, t = lane & 3;
    for (int nt = warp; nt < NT; nt += W) {
        const int u = nt * 8 + g;                // this lane's unit for the B fragment
        float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
        for (int k0 = 0; k0 < KP; k0 += 16) {
            const int ka = k0 + 2 * t, kb = ka + 8;
            uint32_t b0 = 0u, b1 = 0u;
            if (u < UNITS) {
                if (ka < K) b0 = __ldg(reinterpret_cast<const unsigned int*>(w + u * K + ka));
                if (kb < K) b1 = __ldg(reinterpret_cast<const unsigned int*>(w + u * K + kb));
            }
            const uint32_t* xa = X + (ka >> 1) * kActStride;
            const uint32_t* xb = X + (kb >> 1) * kActStride;
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int r = mt * 16 + g;
                mma_bf16_16816(acc[mt], ka < K ? xa[r] : 0u, ka < K ? xa[r + 8] : 0u, kb < K ? xb[r] : 0u,
                               kb < K ? xb[r + 8] : 0u, b0, b1);
            }
        }
        // epilogue: D element (row g (+8), col 2t (+1)) -> unit u0 (+1), replica mt*16 + g (+8)
        const int u0 = nt * 8 + 2 * t;
        const float bb0 = u0 < UNITS ? __bfloat162float(bias[u0]) : 0.f;
        const float bb1 = u0 + 1 < UNITS ? __bfloat162float(bias[u0 + 1]) : 0.f;
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int r = mt * 16 + g;
            float z00 = acc[mt][0] + bb0, z01 = acc[mt][1] + bb1;       // replica r
            float z10 = acc[mt][2] + bb0, z11 = acc[mt][3] + bb1;       // replica r + 8
            if (HIDDEN) {
                uint32_t* Yp = static_cast<uint32_t*>(Y) + (u0 >> 1) * kActStride;
                Yp[r] = pack_bf16x2(tanhf(z00), tanhf(z01));
                Yp[r + 8] = pack_bf16x2(tanhf(z10), tanhf(z11));
            } else {
                float* Yf = static_cast<float*>(Y);
                if (u0 < UNITS) { Yf[u0 * kOutStride + r] = z00; Yf[u0 * kOutStride + r + 8] = z10; }
                if (u0 + 1 < UNITS) { Yf[(u0 + 1) * kOutStride + r] = z01; Yf[(u0 + 1) * kOutStride + r + 8] = z11; }
            }
        }
    }
}

// features (bufA rows 0..3) -> hidden 1 (bufB) -> hidden 2 (bufA) -> outputs
// (bufB, FP32); a barrier after each layer (called by every thread of the CTA).
// Each buffer is read only by the layer after the one that wrote it.
__device__ __forceinline__ void mlp_block(const __nv_bfloat16* __restrict__ w, uint32_t* bufA, uint32_t* bufB,
                                          int warp, int W, int lane) {
    mlp_layer_mma<kMlpIn, kMlpHidden, true>(w + kOffW1, w + kOffB1, bufA, bufB, warp, W, lane);
    __syncthreads();
    mlp_layer_mma<kMlpHidden, kMlpHidden, true>(w + kOffW2, w + kOffB2, bufB, bufA, warp, W, lane);
    __syncthreads();
    mlp_layer_mma<kMlpHidden, kMlpOut, false>(w + kOffW3, w + kOffB3, bufA, bufB, warp, W, lane);
    __syncthreads();
}

// the features of one replica into packed row pairs of bufA (lane = replica)
__device__ __forceinline__ void store_features(uint32_t* bufA, const float* f, int lane) {
#pragma unroll
    for (int kp = 0; kp < kMlpIn / 2; kp++) bufA[kp * kActStride + lane] = pack_bf16x2(f[2 * kp], f[2 * kp + 1]);
}

__device__ __forceinline__ float argf(float2 a) { return atan2f(a.y, a.x); }

// TMA chunks in flight per warp.  Two (one being read, one loading) keep the
// kernel's shared memory under a third of the SM's, so three CTAs of 8 warps
// share an SM (a chunk takes longer to read than to load from L2).
constexpr int kLStages = 2;
// two network buffers of 32 packed rows each (the outputs, 26 FP32 rows of
// kOutStride, fit in one)
constexpr int kMlpBufWords = (kMlpHidden / 2) * kActStride;
static_assert(kMlpOut * kOutStride <= kMlpBufWords, "output rows fit a network buffer");

// amplitudes [N+1][32] float2, partial fields [W][32] float4, TMA rings
// [W][kLStages][kStage] int2, their barriers [W][kLStages], the two network
// buffers, then the roles' exchange rows [kXchRows][32] float
__host__ __device__ inline size_t learned_base_bytes(int N, int warps) {
    return (size_t)(N + 1) * kRepBlock * sizeof(float2) + (size_t)warps * kRepBlock * sizeof(float4) +
           (size_t)warps * kLStages * kStage * sizeof(int2) + (size_t)warps * kLStages * sizeof(uint64_t) +
           (size_t)2 * kMlpBufWords * sizeof(uint32_t) + (size_t)kXchRows * kRepBlock * sizeof(float);
}

// cluster variant: the partial-field exchange buffer [2][C][32] float4 after
// the network buffers, at a 16-byte boundary
__host__ __device__ inline size_t learned_cluster_buffer_offset(int N, int warps) {
    return (learned_base_bytes(N, warps) + 15) & ~(size_t)15;
}

// cluster variant: the exchange buffer, then the cluster's abort flag (one word)
inline size_t learned_smem_bytes(int N, int warps, int C = 1) {
    if (C > 1) return learned_cluster_buffer_offset(N, warps) + (size_t)2 * C * kRepBlock * sizeof(float4) + 16;
    return learned_base_bytes(N, warps);
}

// CL: one replica block over a thread-block cluster of P.cluster CTAs.  Each
// CTA reads 1/C of every list; the partial fields of both passes meet in every
// CTA's exchange buffer (distributed shared memory, one cluster barrier per
// exchange, double-buffered by exchange parity); every CTA then evaluates the
// network and takes the same decision on the same numbers, so the amplitude
// copies stay identical; rank 0 writes records, trace and results.
template <bool CL>
__global__ void __launch_bounds__(256, 3) learned_sweep_kernel(const SweepParams P, const LearnParams L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int C = CL ? P.cluster : 1;
    const uint32_t rank = CL ? cluster_rank() : 0u;
    const bool writer = rank == 0;
    const Unit U = P.units[blockIdx.x / C];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N, R = S.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = P.warps;
    const bool learned = L.mode == 2;
    float2* sp = reinterpret_cast<float2*>(smem_raw);
    float4* red = reinterpret_cast<float4*>(sp + (size_t)(N + 1) * kRepBlock);
    int2* ring_all = reinterpret_cast<int2*>(red + (size_t)W * kRepBlock);
    int2* ring = ring_all + (size_t)warp * kLStages * kStage;
    uint64_t* bars_all = reinterpret_cast<uint64_t*>(ring_all + (size_t)W * kLStages * kStage);
    uint64_t* bars = bars_all + warp * kLStages;
    uint32_t* bufA = reinterpret_cast<uint32_t*>(bars_all + W * kLStages);
    uint32_t* bufB = bufA + kMlpBufWords;
    const float* outs = reinterpret_cast<const float*>(bufB);
    float* xch = reinterpret_cast<float*>(bufB + kMlpBufWords);
    auto out_of = [&](int o) { return outs[o * kOutStride + lane]; };
    float4* cred = CL ? reinterpret_cast<float4*>(smem_raw + learned_cluster_buffer_offset(N, W)) : nullptr;
    int* cflag = CL ? reinterpret_cast<int*>(cred + (size_t)2 * C * kRepBlock) : nullptr;   // cluster abort flag

    const bool active = lane < U.rep_count;
    const int64_t gr = S.rep_off + U.rep_begin + lane;
    for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
        const int site = idx >> 5, l = idx & 31;
        float2 v = make_float2(1.f, 0.f);
        if (l < U.rep_count) v = P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l];
        sp[idx] = v;
    }
    if (threadIdx.x < kRepBlock) sp[N * kRepBlock + threadIdx.x] = make_float2(1.f, 0.f);
    if (CL && threadIdx.x == 0) *cflag = 0;

    double E = 0.0, beta_d = 0.0;
    float beta = 0.f;
    long long nacc = 0, nprop = 0;
    uint32_t k0 = 0, k1 = 0;
    if (active) {                               // every warp may run a sampling role
        const uint64_t key = P.key[gr];
        k0 = (uint32_t)key;
        k1 = (uint32_t)(key >> 32);
    }
    if (warp == 0 && active) {
        E = P.energy[gr];
        beta_d = P.beta[gr];
        beta = (float)beta_d;
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2, total = P.nsweeps * steps;
    Stream<4> st;
    st.key0 = S.pair_key0;
    st.key1 = S.pair_key1;
    st.N = N;
    st.site_chunks = P.site_chunks_g + S.split_off;   // built with the pair sub-lists (set_proposal)
    st.pair_chunks = P.pair_chunks + S.pair_off;
    st.sweep0 = sweep0;
    st.steps = steps;
    st.total = total;
    const int TW = C * W, gw = (int)rank * W + warp;
    st.part0 = gw * (kSplit / TW);
    st.part1 = (gw + 1) * (kSplit / TW);
    if (lane == 0) {
        for (int s = 0; s < kLStages; s++) mbar_init(bars + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_shared();
    }
    __syncwarp();
    Cursor pc = st.first();
    uint32_t issued = 0, consumed = 0;
    bool ok_wait = true;
    auto issue = [&]() {
        if (pc.m >= total) return;
        const uint32_t slot = issued % kLStages;
        if (lane == 0) {
            const int64_t b = __ldg(P.chunk_start + pc.c), e = __ldg(P.chunk_start + pc.c + 1);
            const uint32_t bytes = (uint32_t)((e - b) * sizeof(int2));
            mbar_expect_tx(bars + slot, bytes);
            bulk_g2s(ring + slot * kStage, P.entries + b, bytes, bars + slot);
        }
        issued++;
        st.next(pc);
    };
    for (int s = 0; s < kLStages; s++) issue();
    __shared__ __align__(8) uint64_t stall_bar;      // test hook: nothing arrives on it
    if (threadIdx.x == 0 && P.stall_move >= 0) {
        mbar_init(&stall_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (CL) cluster_sync();                    // every CTA runs before the first remote store
    uint32_t xchg = 0;                         // exchanges so far (buffer parity)
    bool aborted = false;                      // set uniformly over the CTA (cluster) by reduce()

    // one pass over this warp's share of two lists: the sites' lists (base 0;
    // tiles, or the group format built with the pair sub-lists) or the pair's
    // sub-lists (base 2, group format)
    auto pass = [&](int m, int base, float* h) {
        for (int which = base; which < base + 2 && ok_wait; which++) {
            int c, c_end;
            st.range(m, which, c, c_end);
            for (; c < c_end; c++) {
                const uint32_t slot = consumed % kLStages;
                ok_wait = ring_wait(bars + slot, (consumed / kLStages) & 1u, P.status, P.wait_clocks);
                if (!ok_wait) break;               // stop consuming and issuing; abort in reduce()
                const int n = (int)(__ldg(P.chunk_start + c + 1) - __ldg(P.chunk_start + c));
                const int k2 = 2 * (which & 1);
                if (which < 2 && S.fc_tiles)      // unrolled by 2: the kernel is held to 80 registers
                    accumulate_tiles<2>(ring + slot * kStage, n, sp, lane, h[k2], h[k2 + 1]);
                else accumulate_chunk(ring + slot * kStage, n, sp, lane, h[k2], h[k2 + 1]);
                consumed++;
                __syncwarp();
                if (lane == 0) fence_async_shared();
                issue();
            }
        }
    };
    // partial sums of all warps (and all CTAs of the cluster) -> warp 0.
    // Also agrees on an abort: a warp whose wait ran out makes the whole CTA
    // (and, through the flag, the whole cluster) set `aborted` here.
    auto reduce = [&](const float* h) {
        red[warp * kRepBlock + lane] = make_float4(h[0], h[1], h[2], h[3]);
        const bool bad = __syncthreads_or(!ok_wait);
        float4 hs = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!CL && bad) {
            aborted = true;
            return hs;
        }
        if (warp == 0)
            for (int w = 0; w < W; w++) {
                const float4 v = red[w * kRepBlock + lane];
                hs.x += v.x; hs.y += v.y; hs.z += v.z; hs.w += v.w;
            }
        if (CL) {
            float4* buf = cred + (size_t)(xchg & 1u) * C * kRepBlock;
            if (warp == 0) {
                for (int q = 0; q < C; q++) st_cluster_f4(buf + rank * kRepBlock + lane, (uint32_t)q, hs);
                if (bad && lane == 0)
                    for (int q = 0; q < C; q++) st_cluster_u32(cflag, (uint32_t)q, 1u);
            }
            cluster_sync();
            if (*(volatile int*)cflag) {
                aborted = true;
                return hs;
            }
            if (warp == 0) {
                hs = buf[lane];
                for (int q = 1; q < C; q++) {
                    const float4 v = buf[q * kRepBlock + lane];
                    hs.x += v.x; hs.y += v.y; hs.z += v.z; hs.w += v.w;
                }
            }
            xchg++;
        }
        return hs;
    };

    for (int m = 0; m < total; m++) {
        const long long sw = sweep0 + m / steps;
        const int k = m % steps;
        int i0, j0;
        pair_pick(S.pair_key0, S.pair_key1, (uint64_t)sw, (uint32_t)k, N, i0, j0);

        // ---- fields at x: h_i (with a_j), h_j (with a_i) ---------------------------
        float h[4] = {0.f, 0.f, 0.f, 0.f};
        if (m == P.stall_move) ok_wait = stall_wait(&stall_bar, P.status, P.wait_clocks);
        pass(m, 0, h);
        const float4 hs1 = reduce(h);
        if (aborted) break;
        float2 ai = make_float2(0.f, 0.f), aj = ai, ain = ai, ajn = ai;
        const float2 hi1 = make_float2(hs1.x, hs1.y), hj1 = make_float2(hs1.z, hs1.w);
        float cu = 0.f, lq_fwd = 0.f, lq_ratio = 0.f, tn = 0.5f, psi_i = 0.f, psi_j = 0.f, Ssum = 1.f;
        bool ok = true;
        MoveStream g = role_stream(k0, k1, (uint32_t)k, (uint64_t)sw, kAcceptBlock);   // accept and record draws
        if (warp == 0) {
            ai = sp[i0 * kRepBlock + lane];
            aj = sp[j0 * kRepBlock + lane];
            Ssum = fmaf(ai.x, ai.x, ai.y * ai.y) + fmaf(aj.x, aj.x, aj.y * aj.y);
            if (learned) {
                float f[kMlpIn];
                pair_features(ai, aj, hi1, hj1, beta, f);
                store_features(bufA, f, lane);
            }
        }
        // ---- proposal -------------------------------------------------------------
        if (learned) {
            __syncthreads();
            mlp_block(L.w, bufA, bufB, warp, W, lane);
            for (int r = warp; r < kRoles; r += W) learned_role(r, true, out_of, xch, lane, k0, k1, (uint32_t)k, sw);
            __syncthreads();
        }
        if (warp == 0) {
            if (!learned) {
                const U4 w = move_words(k0, k1, (uint64_t)sw, (uint32_t)k);
                propose<0>(ai, aj, w, ain, ajn);
                cu = u01f(w.w);
                tn = fmaf(ain.x, ain.x, ain.y * ain.y) / Ssum;
                psi_i = argf(ain) + argf(hi1);
                psi_j = argf(ajn) + argf(hj1);
            } else {
                // the roles' draws: t' = X/(X+Y) inside (kTEdge, 1 - kTEdge) and
                // both phases, else the move is rejected
                const float X = xch[X_X * 32 + lane], Y = xch[X_Y * 32 + lane];
                ok = X >= 0.f && Y >= 0.f && X + Y > 0.f && xch[X_OK0 * 32 + lane] != 0.f &&
                     xch[X_OK1 * 32 + lane] != 0.f;
                if (ok) {
                    tn = X / (X + Y);
                    ok = tn > kTEdge && tn < 1.0f - kTEdge;
                }
                if (ok) {
                    psi_i = xch[X_PSI0 * 32 + lane];
                    psi_j = xch[X_PSI1 * 32 + lane];
                    const float mi = sqrtf(Ssum * tn), mj = sqrtf(Ssum * (1.0f - tn));
                    float s1, c1, s2, c2;
                    sincosf(psi_i - argf(hi1), &s1, &c1);
                    sincosf(psi_j - argf(hj1), &s2, &c2);
                    ain = make_float2(mi * c1, mi * s1);
                    ajn = make_float2(mj * c2, mj * s2);
                    // log q_L(x'|x) = log Beta + both mixtures, as log_learned_density
                    lq_fwd = log_beta_pdf_lg(tn, xch[X_A * 32 + lane], xch[X_B * 32 + lane], xch[X_LGA * 32 + lane],
                                             xch[X_LGB * 32 + lane], xch[X_LGAB * 32 + lane]) +
                             xch[X_VM0 * 32 + lane] + xch[X_VM1 * 32 + lane] - log_plain_density(tn);
                } else {
                    ain = ai;
                    ajn = aj;
                }
                cu = g.uniform();
            }
            // the pair's slots hold the changes while the sub-lists are read:
            // every term there contains exactly one of a_i, a_j (linearly or
            // conjugated), so the sums are h_i(x') - h_i(x) and h_j(x') - h_j(x)
            sp[i0 * kRepBlock + lane] = make_float2(ain.x - ai.x, ain.y - ai.y);
            sp[j0 * kRepBlock + lane] = make_float2(ajn.x - aj.x, ajn.y - aj.y);
        }
        __syncthreads();

        // ---- field changes from the pair's sub-lists --------------------------------
        h[0] = h[1] = h[2] = h[3] = 0.f;
        pass(m, 2, h);
        const float4 dh = reduce(h);
        if (aborted) break;
        float dE = 0.f;
        float2 hi2 = hi1, hj2 = hj1;
        if (warp == 0) {
            hi2 = make_float2(hi1.x + dh.x, hi1.y + dh.y);
            hj2 = make_float2(hj1.x + dh.z, hj1.y + dh.w);
            const float dix = ain.x - ai.x, diy = ain.y - ai.y, djx = ajn.x - aj.x, djy = ajn.y - aj.y;
            dE = -fmaf(dix, hi2.x, -diy * hi2.y) - fmaf(djx, hj1.x, -djy * hj1.y);
            if (learned) {
                float f[kMlpIn];
                pair_features(ain, ajn, hi2, hj2, beta, f);
                store_features(bufA, f, lane);
                // the reverse move's phases, measured from the fields at x'
                xch[X_PSI0 * 32 + lane] = argf(ai) + argf(hi2);
                xch[X_PSI1 * 32 + lane] = argf(aj) + argf(hj2);
            }
        }
        if (learned) {
            __syncthreads();
            mlp_block(L.w, bufA, bufB, warp, W, lane);
            for (int r = warp; r < kRoles; r += W) learned_role(r, false, out_of, xch, lane, k0, k1, (uint32_t)k, sw);
            __syncthreads();
        }
        if (warp == 0) {
            bool accept;
            if (!learned) {
                if (beta_d == 0.0) accept = true;
                else accept = (dE <= 0.f) || (cu < expf(-beta * dE));
            } else {
                // The sampler proposes t' only inside I = (1e-7, 1 - 1e-7), so the
                // move's density is q_L 1[t' in I]; the reverse move exists only
                // if the current t is in I as well.  Accepting only then gives
                // the transition density min(pi q_L, pi' q_L') 1[t in I] 1[t' in I],
                // symmetric in x and x'.
                const float t = fmaf(ai.x, ai.x, ai.y * ai.y) / Ssum;
                const bool t_in = t > kTEdge && t < 1.0f - kTEdge;
                if (t_in) {
                    const float lq_rev = log_beta_pdf_lg(t, xch[X_A * 32 + lane], xch[X_B * 32 + lane],
                                                         xch[X_LGA * 32 + lane], xch[X_LGB * 32 + lane],
                                                         xch[X_LGAB * 32 + lane]) +
                                         xch[X_VM0 * 32 + lane] + xch[X_VM1 * 32 + lane] - log_plain_density(t);
                    lq_ratio = lq_rev - lq_fwd;
                }
                accept = ok && t_in && (logf(cu) < -beta * dE + lq_ratio);
            }
            sp[i0 * kRepBlock + lane] = accept ? ain : ai;
            sp[j0 * kRepBlock + lane] = accept ? ajn : aj;
            if (accept) {
                E += (double)dE;
                nacc++;
            }
            nprop++;
            if (!learned && accept && active && writer && L.records != nullptr && u01f(g.next()) < L.rec_prob) {
                float f[kMlpIn];
                pair_features(ai, aj, hi1, hj1, beta, f);
                const unsigned long long slot = atomicAdd(L.rec_count, 1ull) % (unsigned long long)L.rec_cap;
                float* rec = L.records + slot * kRecordFloats;
                for (int q = 0; q < kMlpIn; q++) rec[q] = f[q];
                // t' within float range of (0, 1): log t' and log(1-t') stay finite
                rec[kMlpIn] = fminf(fmaxf(tn, 1e-6f), 1.0f - 1e-6f);
                rec[kMlpIn + 1] = psi_i;
                rec[kMlpIn + 2] = psi_j;
            }
            if (writer && P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + lane == P.trace_rep &&
                active) {
                const long long idx = (sw - P.trace_sweep0) * steps + k;
                if (idx >= 0 && idx < P.trace_cap) {
                    pspin_move_record* r = reinterpret_cast<pspin_move_record*>(P.trace) + idx;
                    r->i0 = i0; r->j0 = j0;
                    r->ai_old[0] = ai.x; r->ai_old[1] = ai.y; r->aj_old[0] = aj.x; r->aj_old[1] = aj.y;
                    r->ai_new[0] = ain.x; r->ai_new[1] = ain.y; r->aj_new[0] = ajn.x; r->aj_new[1] = ajn.y;
                    r->dE = dE;
                    r->accepted = accept ? 1 : 0;
                    r->log_q_ratio = lq_ratio;
                    r->log_u = logf(cu);
                }
            }
        }
        __syncthreads();
    }
    if (aborted) drain_ring(bars, kLStages, consumed, issued, P.status);   // state stays as before the launch
    if (writer && !aborted) {
        for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
            const int site = idx >> 5, l = idx & 31;
            if (l < U.rep_count) P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l] = sp[idx];
        }
        if (warp == 0 && active) {
            P.energy[gr] = E;
            P.accepted[gr] += nacc;
            P.proposed[gr] += nprop;
        }
    }
    if (CL) cluster_sync();                    // no CTA leaves while a remote store may target it
}

size_t learned_smem_bytes_host(int N, int warps, int C) { return learned_smem_bytes(N, warps, C); }

// max_clusters != null (clusters only): reports how many clusters of this
// shape can be resident instead of launching (0: the shape does not fit)
cudaError_t launch_learned_sweep(const SweepParams& p, const LearnParams& l, int n_units, int max_N,
                                 cudaStream_t st, int* max_clusters) {
    if (n_units <= 0) return cudaSuccess;
    if (p.pair_chunks == nullptr && max_clusters == nullptr) return cudaErrorInvalidValue;
    const int C = p.cluster > 1 ? p.cluster : 1;
    if (C > 16 || (kSplit % (C * p.warps)) != 0) return cudaErrorInvalidValue;
    const size_t smem = learned_smem_bytes(max_N, p.warps, C);
    if (C == 1) {
        cudaError_t e = cudaFuncSetAttribute(learned_sweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        learned_sweep_kernel<false><<<n_units, 32 * p.warps, smem, st>>>(p, l);
        return cudaGetLastError();
    }
    auto kern = learned_sweep_kernel<true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && C > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(n_units * C));
    cfg.blockDim = dim3((unsigned)(32 * p.warps));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (max_clusters) return cudaOccupancyMaxActiveClusters(max_clusters, kern, &cfg);
    e = cudaLaunchKernelEx(&cfg, kern, p, l);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// ------------------------------------------------------------------ training
// Per record: forward and backward through the network (FP32 master
// weights); activations and deltas saved for the per-parameter reduction.
constexpr int kSaveFloats = kMlpIn + 2 * kMlpHidden + 2 * kMlpHidden + kMlpOut;   // f, h1, h2, d1, d2, d3

__global__ void mlp_fwd_bwd_kernel(const float* __restrict__ w, const float* __restrict__ records,
                                   const int* __restrict__ index, int n, float* __restrict__ save,
                                   float* __restrict__ loss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const float* rec = records + (int64_t)(index ? index[b] : b) * kRecordFloats;
    float* sv = save + (int64_t)b * kSaveFloats;
    float* f = sv;
    float* h1 = f + kMlpIn;
    float* h2 = h1 + kMlpHidden;
    float* d1 = h2 + kMlpHidden;
    float* d2 = d1 + kMlpHidden;
    float* d3 = d2 + kMlpHidden;
    for (int i = 0; i < kMlpIn; i++) f[i] = rec[i];
    float out[kMlpOut];
    mlp_forward_rows(w, f, h1, h2, out);
    loss[b] = loss_output_grad(out, rec[kMlpIn], rec[kMlpIn + 1], rec[kMlpIn + 2], d3);
    for (int i = 0; i < kMlpHidden; i++) {
        float s = 0.f;
        for (int o = 0; o < kMlpOut; o++) s = fmaf(w[kOffW3 + o * kMlpHidden + i], d3[o], s);
        d2[i] = s * (1.0f - h2[i] * h2[i]);
    }
    for (int i = 0; i < kMlpHidden; i++) {
        float s = 0.f;
        for (int o = 0; o < kMlpHidden; o++) s = fmaf(w[kOffW2 + o * kMlpHidden + i], d2[o], s);
        d1[i] = s * (1.0f - h1[i] * h1[i]);
    }
}

// gradient of the mean loss, one thread per parameter, summed over records
// in a fixed order (deterministic)
__global__ void mlp_grad_reduce_kernel(const float* __restrict__ save, int n, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    // saved layout per record: f | h1 | h2 | d1 | d2 | d3
    constexpr int F0 = 0, H1 = kMlpIn, H2 = H1 + kMlpHidden, D1 = H2 + kMlpHidden, D2 = D1 + kMlpHidden,
                  D3 = D2 + kMlpHidden;
    int dofs, aofs = 0, ai = -1;   // delta index; activation index (ai < 0: bias)
    if (p < kOffB1) { dofs = D1 + p / kMlpIn; aofs = F0; ai = p % kMlpIn; }
    else if (p < kOffW2) { dofs = D1 + (p - kOffB1); }
    else if (p < kOffB2) { const int q = p - kOffW2; dofs = D2 + q / kMlpHidden; aofs = H1; ai = q % kMlpHidden; }
    else if (p < kOffW3) { dofs = D2 + (p - kOffB2); }
    else if (p < kOffB3) { const int q = p - kOffW3; dofs = D3 + q / kMlpHidden; aofs = H2; ai = q % kMlpHidden; }
    else { dofs = D3 + (p - kOffB3); }
    float s = 0.f;
    for (int b = 0; b < n; b++) {
        const float* sv = save + (int64_t)b * kSaveFloats;
        s = fmaf(sv[dofs], ai >= 0 ? sv[aofs + ai] : 1.0f, s);
    }
    grad[p] = s / (float)n;
}

__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, __nv_bfloat16* __restrict__ wbf, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp, vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float wp = w[p] - lr * (mp / c1) / (sqrtf(vp / c2) + eps);
    w[p] = wp;
    wbf[p] = __float2bfloat16_rn(wp);
}

__global__ void to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wbf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kMlpParams) wbf[p] = __float2bfloat16_rn(w[p]);
}

__global__ void sample_index_kernel(int* __restrict__ idx, int n, unsigned long long filled, uint32_t k0, uint32_t k1,
                                    uint32_t step) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const U4 r = philox4x32_10(U4{(uint32_t)b, step, 0x74726e00u, 0u}, k0, k1);
    idx[b] = (int)(((uint64_t)r.x * filled) >> 32);
}

cudaError_t launch_mlp_fwd_bwd(const float* w, const float* records, const int* index, int n, float* save,
                               float* loss, cudaStream_t st) {
    mlp_fwd_bwd_kernel<<<(n + 127) / 128, 128, 0, st>>>(w, records, index, n, save, loss);
    return cudaGetLastError();
}
cudaError_t launch_mlp_grad(const float* save, int n, float* grad, cudaStream_t st) {
    mlp_grad_reduce_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(save, n, grad);
    return cudaGetLastError();
}
cudaError_t launch_adam(float* w, float* m, float* v, const float* g, __nv_bfloat16* wbf, float lr, int t,
                        cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(w, m, v, g, wbf, lr, b1, b2, 1e-8f,
                                                          1.0f - powf(b1, (float)t), 1.0f - powf(b2, (float)t));
    return cudaGetLastError();
}
cudaError_t launch_to_bf16(const float* w, __nv_bfloat16* wbf, cudaStream_t st) {
    to_bf16_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(w, wbf);
    return cudaGetLastError();
}
cudaError_t launch_sample_index(int* idx, int n, unsigned long long filled, uint64_t key, uint32_t step,
                                cudaStream_t st) {
    sample_index_kernel<<<(n + 255) / 256, 256, 0, st>>>(idx, n, filled, (uint32_t)key, (uint32_t)(key >> 32), step);
    return cudaGetLastError();
}

}  // namespace pspin
