// sweep_multi.cu -- the plain pair-rotation sweep with K replicas per lane:
// one unit is 32K replicas of one sample (replica k*32 + lane of the unit in
// lane `lane`, slot k), split over a cluster of C CTAs of W warps (C = 1: one
// CTA, no cluster).
//
// Same moves, RNG streams and Metropolis rule as sweep_kernel and
// sweep_cluster_kernel, organised as the latter (one barrier per move, every
// warp decides, all warps precompute the random parts of a window of moves
// a window ahead).
// What K changes: every staged coupling, broadcast from shared memory, is
// used for the lane's K replicas, so per FFMA there are K times fewer
// coupling loads, K times more independent accumulator chains per warp, and
// K times fewer move barriers per replica.  The amplitudes are stored
// [site][K][32] float2.
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

constexpr int kWinK = 4;   // moves per window of precomputed proposal parts

// Shared memory of one CTA: amplitudes [(N+1)][K][32] float2; TMA rings
// [W][kStages][kStage] int2; ring mbarriers [W][kStages]; the precomputed
// proposal parts [2][kWinK][7][K][32] float; at a 16-byte boundary the
// exchange buffer [2][C*W][K][32] float4 and the cluster's abort flag.
__host__ __device__ inline size_t multi_pre_offset(int N, int W, int K) {
    return (size_t)(N + 1) * K * kRepBlock * sizeof(float2) + (size_t)W * kStages * kStage * sizeof(int2) +
           (size_t)W * kStages * sizeof(uint64_t);
}
__host__ __device__ inline size_t multi_buffer_offset(int N, int W, int K) {
    return (multi_pre_offset(N, W, K) + (size_t)2 * kWinK * 7 * K * kRepBlock * sizeof(float) + 15) & ~(size_t)15;
}
inline size_t multi_smem_bytes(int N, int W, int C, int K) {   // + the static ring tags
    return multi_buffer_offset(N, W, K) + (size_t)2 * C * W * K * kRepBlock * sizeof(float4) + 16 + kStaticSmem;
}


template <int VARIANT, int K>
__global__ void __launch_bounds__(256, 1) sweep_multi_kernel(const SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int C = P.cluster;
    const uint32_t rank = C > 1 ? cluster_rank() : 0u;
    const Unit U = P.units[blockIdx.x / C];    // rep_count <= 32 K
    const SampleDev S = P.samples[U.sample];
    const int N = S.N, R = S.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int W = P.warps, CW = C * W;
    const int KB = K * kRepBlock;              // replicas of the unit
    float2* sp = reinterpret_cast<float2*>(smem_raw);                              // [(N+1)][K][32]
    int2* ring_all = reinterpret_cast<int2*>(sp + (size_t)(N + 1) * KB);
    int2* ring = ring_all + (size_t)warp * kStages * kStage;
    uint64_t* bars_all = reinterpret_cast<uint64_t*>(ring_all + (size_t)W * kStages * kStage);
    uint64_t* bars = bars_all + warp * kStages;
    float* pre = reinterpret_cast<float*>(smem_raw + multi_pre_offset(N, W, K));      // [2][kWinK][7][K][32]
    float4* cred = reinterpret_cast<float4*>(smem_raw + multi_buffer_offset(N, W, K)); // [2][C*W][K][32]
    int* cflag = reinterpret_cast<int*>(cred + (size_t)2 * CW * KB);
    const bool writer = rank == 0;

    load_block_amplitudes(sp, P.spins + S.spin_off + U.rep_begin, R, N, KB, U.rep_count);   // column k*32 + lane
    for (int idx = threadIdx.x; idx < KB; idx += blockDim.x) sp[(size_t)N * KB + idx] = make_float2(1.f, 0.f);
    if (threadIdx.x == 0) *cflag = 0;

    double E[K], beta_d[K];
    float beta[K];
    int nacc[K], nprop[K];
    uint32_t k0[K], k1[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        E[k] = 0.0;
        beta_d[k] = 0.0;
        beta[k] = 0.f;
        nacc[k] = nprop[k] = 0;
        k0[k] = k1[k] = 0;
        const int rr = k * kRepBlock + lane;
        if (rr < U.rep_count) {
            const int64_t gr = S.rep_off + U.rep_begin + rr;
            beta_d[k] = P.beta[gr];
            beta[k] = (float)beta_d[k];
            const uint64_t key = P.key[gr];
            k0[k] = (uint32_t)key;
            k1[k] = (uint32_t)(key >> 32);
            if (warp == 0) E[k] = P.energy[gr];
        }
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2, total = P.nsweeps * steps;
    const int gw = (int)rank * W + warp;

    Stream<2, false> st;
    st.key0 = S.pair_key0;
    st.key1 = S.pair_key1;
    st.N = N;
    st.site_chunks = P.site_chunks + S.split_off;
    st.pair_chunks = nullptr;
    st.sweep0 = sweep0;
    st.steps = steps;
    st.total = total;
    st.part0 = gw * (kSplit / CW);
    st.part1 = (gw + 1) * (kSplit / CW);
    if (lane == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(bars + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_shared();
    }
    __syncwarp();
    Cursor pc = st.first();
    uint32_t issued = 0, consumed = 0;
    bool ok = true;
    // each ring slot's tag: {move * 2 + list, entries}, written by lane 0 when
    // the copy is issued, so the consumer needs no list lookups of its own
    __shared__ int2 rtag_all[8 * kStages];
    int2* rtag = rtag_all + warp * kStages;
    auto issue = [&]() {
        if (pc.m >= total) return;
        const uint32_t slot = issued % kStages;
        if (lane == 0) {
            const int64_t b = __ldg(P.chunk_start + pc.c), e = __ldg(P.chunk_start + pc.c + 1);
            const uint32_t bytes = (uint32_t)((e - b) * sizeof(int2));
            rtag[slot] = make_int2(pc.m * 2 + pc.which, (int)(e - b));
            mbar_expect_tx(bars + slot, bytes);
            bulk_g2s(ring + slot * kStage, P.entries + b, bytes, bars + slot);
        }
        issued++;
        st.next(pc);
    };
    for (int s = 0; s < kStages; s++) issue();

    // random words, sines and cosines of the moves of window wn for the
    // lane's K replicas, shared out over the CTA's warps, into pre[wn & 1]
    auto make_window = [&](int wn) {
        for (int t = warp; t < kWinK; t += W) {
            const int m = wn * kWinK + t;
            if (m >= total) break;
            const long long sw = sweep0 + m / steps;
            float* dst = pre + ((wn & 1) * kWinK + t) * 7 * KB;
#pragma unroll
            for (int k = 0; k < K; k++) {
                float tt[7];
                move_trig<VARIANT>(move_words(k0[k], k1[k], (uint64_t)sw, (uint32_t)(m % steps)), tt);
#pragma unroll
                for (int q = 0; q < 7; q++) dst[(q * K + k) * kRepBlock + lane] = tt[q];
            }
        }
    };
    auto pair_of = [&](int m, int& i0, int& j0) {
        pair_pick(S.pair_key0, S.pair_key1, (uint64_t)(sweep0 + m / steps), (uint32_t)(m % steps), N, i0, j0);
    };
    int ci0 = 0, cj0 = 0;
    float2 cai[K], caj[K], cain[K], cajn[K];
    float cu[K];
    auto take_pre = [&](int m, int k, float2 ai, float2 aj) {
        const float* src = pre + (((m / kWinK) & 1) * kWinK + m % kWinK) * 7 * KB;
        float t[7];
#pragma unroll
        for (int q = 0; q < 7; q++) t[q] = src[(q * K + k) * kRepBlock + lane];
        cai[k] = ai;
        caj[k] = aj;
        propose_with<VARIANT>(ai, aj, t, cain[k], cajn[k]);
        cu[k] = t[6];
    };

    __shared__ __align__(8) uint64_t stall_bar;      // test hook: nothing arrives on it
    if (threadIdx.x == 0 && P.stall_move >= 0) {
        mbar_init(&stall_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    make_window(0);
    make_window(1);
    __syncthreads();
    if (total > 0) {
        pair_of(0, ci0, cj0);
#pragma unroll
        for (int k = 0; k < K; k++) {
            take_pre(0, k, sp[(ci0 * K + k) * kRepBlock + lane], sp[(cj0 * K + k) * kRepBlock + lane]);
            sp[(cj0 * K + k) * kRepBlock + lane] = cajn[k];   // h_i is evaluated at the proposed a_j
        }
    }
    if (C > 1) cluster_sync();                 // every CTA runs before the first remote store
    else __syncthreads();

    bool aborted = false;
    for (int m = 0; m < total; m++) {
        // window w+1 during the first move of window w (its buffer's last
        // reader is behind barrier kWinK*w - 1)
        if (m >= kWinK && m % kWinK == 0) make_window(m / kWinK + 1);
        // ---- field pass m
        float hix[K], hiy[K], hjx[K], hjy[K];
#pragma unroll
        for (int k = 0; k < K; k++) hix[k] = hiy[k] = hjx[k] = hjy[k] = 0.f;
        if (m == P.stall_move) ok = stall_wait(&stall_bar, P.status, P.wait_clocks);
        // the ring's chunks tagged with move m, in issue order: site i0's list, then j0's
        while (ok) {
            __syncwarp();
            if (consumed == issued) break;
            const uint32_t slot = consumed % kStages;
            const int2 tg = rtag[slot];
            if ((tg.x >> 1) != m) break;
            ok = ring_wait(bars + slot, (consumed / kStages) & 1u, P.status, P.wait_clocks);
            if (!ok) break;
            if ((tg.x & 1) == 0) {
                if (S.fc_tiles) accumulate_tiles_k<K, 4>(ring + slot * kStage, tg.y, sp, lane, hix, hiy);
                else accumulate_records_k<K>(ring + slot * kStage, tg.y, sp, lane, hix, hiy);
            } else {
                if (S.fc_tiles) accumulate_tiles_k<K, 4>(ring + slot * kStage, tg.y, sp, lane, hjx, hjy);
                else accumulate_records_k<K>(ring + slot * kStage, tg.y, sp, lane, hjx, hjy);
            }
            consumed++;
            __syncwarp();
            if (lane == 0) fence_async_shared();
            issue();
        }
        // the next move's pair and its sites' amplitudes in the state the field
        // pass read (move m's decision can change only ci0, cj0)
        int ni0 = 0, nj0 = 0;
        float2 nai[K], naj[K];
        if (m + 1 < total) {
            pair_of(m + 1, ni0, nj0);
#pragma unroll
            for (int k = 0; k < K; k++) {
                nai[k] = sp[(ni0 * K + k) * kRepBlock + lane];
                naj[k] = sp[(nj0 * K + k) * kRepBlock + lane];
            }
        }
        // ---- partials to every CTA (or this one), one barrier
        float4* buf = cred + (size_t)(m & 1) * CW * KB;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float4 mine = make_float4(hix[k], hiy[k], hjx[k], hjy[k]);
            float4* slot = buf + (size_t)(gw * K + k) * kRepBlock + lane;
            if (C > 1) {
                for (int q = 0; q < C; q++) st_cluster_f4(slot, (uint32_t)q, mine);
            } else {
                *slot = mine;
            }
        }
        if (C > 1) {
            if (!ok && lane == 0)
                for (int q = 0; q < C; q++) st_cluster_u32(cflag, (uint32_t)q, 1u);
            cluster_sync();
            if (*(volatile int*)cflag) {
                aborted = true;
                break;
            }
        } else if (__syncthreads_or(!ok)) {
            aborted = true;
            break;
        }
        // ---- decision m for the lane's K replicas, the same in every warp
        float2 ai_post[K], aj_post[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float4 hs = sum_partials(buf + (size_t)k * kRepBlock + lane, C, W, K * kRepBlock);
            const float dix = cain[k].x - cai[k].x, diy = cain[k].y - cai[k].y;
            const float djx = cajn[k].x - caj[k].x, djy = cajn[k].y - caj[k].y;
            const float dE = -fmaf(dix, hs.x, -diy * hs.y) - fmaf(djx, hs.z, -djy * hs.w);
            bool accept;
            if (beta_d[k] == 0.0) accept = true;
            else accept = (dE <= 0.f) || (cu[k] < expf(-beta[k] * dE));
            ai_post[k] = accept ? cain[k] : cai[k];
            aj_post[k] = accept ? cajn[k] : caj[k];
            if (warp == 0) {
                if (accept) {
                    E[k] += (double)dE;
                    nacc[k]++;
                }
                nprop[k]++;
                const int rr = k * kRepBlock + lane;
                if (writer && P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + rr == P.trace_rep &&
                    rr < U.rep_count) {
                    const long long sw = sweep0 + m / steps;
                    const long long idx = (sw - P.trace_sweep0) * steps + m % steps;
                    if (idx >= 0 && idx < P.trace_cap) {
                        pspin_move_record* rec = reinterpret_cast<pspin_move_record*>(P.trace) + idx;
                        rec->i0 = ci0; rec->j0 = cj0;
                        rec->ai_old[0] = cai[k].x; rec->ai_old[1] = cai[k].y;
                        rec->aj_old[0] = caj[k].x; rec->aj_old[1] = caj[k].y;
                        rec->ai_new[0] = cain[k].x; rec->ai_new[1] = cain[k].y;
                        rec->aj_new[0] = cajn[k].x; rec->aj_new[1] = cajn[k].y;
                        rec->dE = dE;
                        rec->accepted = accept ? 1 : 0;
                        rec->log_q_ratio = 0.f;
                        rec->log_u = logf(cu[k]);
                    }
                }
            }
        }
        // ---- proposal m+1 and the final values of the state it reads
        if (m + 1 < total) {
            const int pi0 = ci0, pj0 = cj0;
            ci0 = ni0;
            cj0 = nj0;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const float2 ai1 = ni0 == pi0 ? ai_post[k] : (ni0 == pj0 ? aj_post[k] : nai[k]);
                const float2 aj1 = nj0 == pi0 ? ai_post[k] : (nj0 == pj0 ? aj_post[k] : naj[k]);
                take_pre(m + 1, k, ai1, aj1);
                sp[(pi0 * K + k) * kRepBlock + lane] = pi0 == cj0 ? cajn[k] : ai_post[k];
                sp[(pj0 * K + k) * kRepBlock + lane] = pj0 == cj0 ? cajn[k] : aj_post[k];
                sp[(cj0 * K + k) * kRepBlock + lane] = cajn[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) {
                sp[(ci0 * K + k) * kRepBlock + lane] = ai_post[k];
                sp[(cj0 * K + k) * kRepBlock + lane] = aj_post[k];
            }
        }
    }
    if (aborted) drain_ring(bars, kStages, consumed, issued, P.status);   // state stays as before the launch
    __syncthreads();
    if (writer && !aborted) {
        for (int idx = threadIdx.x; idx < N * KB; idx += blockDim.x) {
            const int site = idx / KB, rr = idx % KB;
            if (rr < U.rep_count) P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + rr] = sp[idx];
        }
        if (warp == 0) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                const int rr = k * kRepBlock + lane;
                if (rr < U.rep_count) {
                    const int64_t gr = S.rep_off + U.rep_begin + rr;
                    P.energy[gr] = E[k];
                    P.accepted[gr] += nacc[k];
                    P.proposed[gr] += nprop[k];
                }
            }
        }
    }
    if (C > 1) cluster_sync();                 // no CTA leaves while a remote store may target it
}

template <int VARIANT, int K>
static cudaError_t launch_multi_one(const SweepParams& p, int n_units, size_t smem, cudaStream_t st, int* max_clusters) {
    auto kern = sweep_multi_kernel<VARIANT, K>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && p.cluster > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(n_units * p.cluster));
    cfg.blockDim = dim3((unsigned)(32 * p.warps));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)p.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = p.cluster > 1 ? 1 : 0;
    if (max_clusters) {
        if (p.cluster > 1) return cudaOccupancyMaxActiveClusters(max_clusters, kern, &cfg);
        int blocks = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, 32 * p.warps, smem);
        *max_clusters = blocks;
        return e;
    }
    e = cudaLaunchKernelEx(&cfg, kern, p);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// units of up to 32K replicas; max_clusters != null: only report how many
// clusters (CTAs when cluster = 1) of this shape can be resident
cudaError_t launch_sweep_multi(const SweepParams& p, int n_units, int variant, int max_N, int K, cudaStream_t st,
                               int* max_clusters) {
    if (n_units <= 0) return cudaSuccess;
    if (p.cluster < 1 || p.cluster > 16 || (kSplit % (p.cluster * p.warps)) != 0) return cudaErrorInvalidValue;
    const size_t smem = multi_smem_bytes(max_N, p.warps, p.cluster, K);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    if (K == 2) return variant == 0 ? launch_multi_one<0, 2>(p, n_units, smem, st, max_clusters)
                                    : launch_multi_one<1, 2>(p, n_units, smem, st, max_clusters);
    if (K == 3) return variant == 0 ? launch_multi_one<0, 3>(p, n_units, smem, st, max_clusters)
                                    : launch_multi_one<1, 3>(p, n_units, smem, st, max_clusters);
    return cudaErrorInvalidValue;
}

size_t multi_smem_bytes_host(int N, int warps, int C, int K) { return multi_smem_bytes(N, warps, C, K); }

}  // namespace pspin
