// sweep_cluster.cu -- the plain pair-rotation sweep with one replica block
// split over a thread-block cluster of C CTAs (C = 2..16).
//
// Same moves, RNG streams and Metropolis rule as sweep_kernel.  Every CTA of
// the cluster holds the block's amplitudes in its own shared memory and
// reads 1/C of every site list through its own TMA rings; the C*W warps of
// the cluster each own kSplit/(C*W) of the 32 parts of a list.
//
// One barrier per move.  A move m is
//   field pass m: every warp accumulates its share of the two sites' fields
//      (with the proposed a_j in j's slot) and stores its float4 partial into
//      slot [rank*W + warp] of every CTA's exchange buffer (distributed
//      shared memory, mapa + st.shared::cluster); then one cluster barrier
//      (release / acquire);
//   decision m: EVERY warp of every CTA sums the C*W partials in the same
//      order (per CTA its warps in order, then the CTAs in rank order) and
//      takes the same Metropolis decision on the same random words, so no
//      warp waits for another to decide or to broadcast;
//   proposal m+1: every warp computes it from the state after the decision
//      and writes the same final values into its lanes' amplitude slots --
//      the decided amplitudes of move m's pair and the proposed a_j of move
//      m+1 -- before its own field pass m+1 reads them.  All writes between
//      two barriers carry the values of the state that the next field pass
//      reads, and each lane reads only its own replica's column, so the
//      warps need no barrier between deciding and reading.
// The state-independent part of a proposal (random words, sines and
// cosines) is computed for windows of kWin moves, a window ahead, by all
// warps of each CTA at once (warp w the window's moves w, w+W, ...), into a
// buffer double-buffered by window, so no warp carries that work alone at
// every move; the exchange buffer is double-buffered by move parity: no warp
// can be more than one move ahead of another (the barrier of each move
// waits for all of them).  Rank 0 writes the results back.
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

constexpr int kWin = 8;    // moves per window of precomputed proposal parts

// Shared memory of one CTA: amplitudes [(N+1)][32] float2; TMA rings
// [W][kStages][kStage] int2; ring mbarriers [W][kStages]; the precomputed
// proposal parts [2][kWin][7][32] float; then, at a 16-byte boundary, the
// exchange buffer [2][C*W][32] float4 and the cluster's abort flag.
__host__ __device__ inline size_t cluster_pre_offset(int N, int warps) {
    return (size_t)(N + 1) * kRepBlock * sizeof(float2) + (size_t)warps * kStages * kStage * sizeof(int2) +
           (size_t)warps * kStages * sizeof(uint64_t);
}
__host__ __device__ inline size_t cluster_buffer_offset(int N, int warps) {
    return (cluster_pre_offset(N, warps) + (size_t)2 * kWin * 7 * kRepBlock * sizeof(float) + 15) & ~(size_t)15;
}
// (+ kStaticSmem: the ring tags are static shared memory, counted here so
// that every fit check against the 227 KB a CTA can have includes them)
inline size_t cluster_smem_bytes(int N, int warps, int C) {
    return cluster_buffer_offset(N, warps) + (size_t)2 * C * warps * kRepBlock * sizeof(float4) + 16 + kStaticSmem;
}


// kBatch: the group records are read in batches whose loads are all in
// flight before their arithmetic (few blocks, so each warp waits on its own
// chain's latency, and a CTA may take every register of an SM); otherwise
// one record at a time, loading a_p, a_o1 once per group (many blocks share
// the SMs at two CTAs each: fewer shared-memory loads, 128 registers).
template <int VARIANT, bool kBatch>
__global__ void __launch_bounds__(256, kBatch ? 1 : 2) sweep_cluster_kernel(const SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int C = P.cluster;
    const uint32_t rank = cluster_rank();
    const Unit U = P.units[blockIdx.x / C];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N;
    const int R = S.R;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int W = P.warps;
    const int CW = C * W;
    float2* sp = reinterpret_cast<float2*>(smem_raw);                          // [(N+1)][32]
    int2* ring_all = reinterpret_cast<int2*>(sp + (size_t)(N + 1) * kRepBlock);
    int2* ring = ring_all + (size_t)warp * kStages * kStage;
    uint64_t* bars_all = reinterpret_cast<uint64_t*>(ring_all + (size_t)W * kStages * kStage);
    uint64_t* bars = bars_all + warp * kStages;
    float* pre = reinterpret_cast<float*>(smem_raw + cluster_pre_offset(N, W));        // [2][kWin][7][32]
    float4* cred = reinterpret_cast<float4*>(smem_raw + cluster_buffer_offset(N, W));  // [2][C*W][32]
    int* cflag = reinterpret_cast<int*>(cred + (size_t)2 * CW * kRepBlock);            // cluster abort flag

    const bool active = lane < U.rep_count;
    const bool writer = rank == 0;
    const int64_t gr = S.rep_off + U.rep_begin + lane;

    load_block_amplitudes(sp, P.spins + S.spin_off + U.rep_begin, R, N, kRepBlock, U.rep_count);
    if (threadIdx.x < kRepBlock) sp[N * kRepBlock + threadIdx.x] = make_float2(1.f, 0.f);  // virtual site
    if (threadIdx.x == 0) *cflag = 0;

    // every warp decides, so every warp holds its lanes' betas
    double E = 0.0, beta_d = 0.0;
    float beta = 0.f;
    long long nacc = 0, nprop = 0;
    uint32_t k0 = 0, k1 = 0;
    if (active) {
        beta_d = P.beta[gr];
        beta = (float)beta_d;
        const uint64_t key = P.key[gr];
        k0 = (uint32_t)key;
        k1 = (uint32_t)(key >> 32);
        if (warp == 0) E = P.energy[gr];
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2;
    const int total = P.nsweeps * steps;
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

    // random words, sines and cosines of the moves of window wn, shared out
    // over the CTA's warps, into pre[wn & 1]
    auto make_window = [&](int wn) {
        for (int t = warp; t < kWin; t += W) {
            const int m = wn * kWin + t;
            if (m >= total) break;
            float tt[7];
            move_trig<VARIANT>(move_words(k0, k1, (uint64_t)(sweep0 + m / steps), (uint32_t)(m % steps)), tt);
            float* dst = pre + ((wn & 1) * kWin + t) * 7 * kRepBlock;
#pragma unroll
            for (int q = 0; q < 7; q++) dst[q * kRepBlock + lane] = tt[q];
        }
    };
    auto pair_of = [&](int m, int& i0, int& j0) {
        pair_pick(S.pair_key0, S.pair_key1, (uint64_t)(sweep0 + m / steps), (uint32_t)(m % steps), N, i0, j0);
    };
    // the pending move (every warp): pair, current and proposed amplitudes, uniform
    int ci0 = 0, cj0 = 0;
    float2 cai = make_float2(0.f, 0.f), caj = cai, cain = cai, cajn = cai;
    float cu = 0.f;
    auto take_pre = [&](int m, float2 ai, float2 aj) {
        const float* src = pre + (((m / kWin) & 1) * kWin + m % kWin) * 7 * kRepBlock;
        float t[7];
#pragma unroll
        for (int q = 0; q < 7; q++) t[q] = src[q * kRepBlock + lane];
        cai = ai;
        caj = aj;
        propose_with<VARIANT>(ai, aj, t, cain, cajn);
        cu = t[6];
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
        take_pre(0, sp[ci0 * kRepBlock + lane], sp[cj0 * kRepBlock + lane]);
        sp[cj0 * kRepBlock + lane] = cajn;     // h_i is evaluated at the proposed a_j
    }
    cluster_sync();                            // every CTA runs before the first remote store

    bool aborted = false;
    for (int m = 0; m < total; m++) {
        // window w+1 during the first move of window w: its buffer's last
        // reader, take_pre at the end of move kWin*w - 2, is behind every
        // warp that has passed barrier kWin*w - 1
        if (m >= kWin && m % kWin == 0) make_window(m / kWin + 1);
        // ---- field pass m
        float h[4] = {0.f, 0.f, 0.f, 0.f};
        if (m == P.stall_move) ok = stall_wait(&stall_bar, P.status, P.wait_clocks);
        // the ring's chunks tagged with move m, in issue order: site i0's list, then j0's
        while (ok) {
            __syncwarp();
            if (consumed == issued) break;
            const uint32_t slot = consumed % kStages;
            const int2 tg = rtag[slot];
            if ((tg.x >> 1) != m) break;
            ok = ring_wait(bars + slot, (consumed / kStages) & 1u, P.status, P.wait_clocks);
            if (!ok) break;                        // stop consuming and issuing; abort below
            if (tg.x & 1) {
                if (S.fc_tiles) accumulate_tiles(ring + slot * kStage, tg.y, sp, lane, h[2], h[3]);
                else if (kBatch) accumulate_records<4>(ring + slot * kStage, tg.y, sp, lane, h[2], h[3]);
                else accumulate_records_1(ring + slot * kStage, tg.y, sp, lane, h[2], h[3]);
            } else {
                if (S.fc_tiles) accumulate_tiles(ring + slot * kStage, tg.y, sp, lane, h[0], h[1]);
                else if (kBatch) accumulate_records<4>(ring + slot * kStage, tg.y, sp, lane, h[0], h[1]);
                else accumulate_records_1(ring + slot * kStage, tg.y, sp, lane, h[0], h[1]);
            }
            consumed++;
            __syncwarp();
            if (lane == 0) fence_async_shared();
            issue();
        }
        // the next move's pair and its sites' amplitudes in the state the
        // field pass just read (this move's decision can change only ci0, cj0)
        int ni0 = 0, nj0 = 0;
        float2 nai = make_float2(0.f, 0.f), naj = nai;
        if (m + 1 < total) {
            pair_of(m + 1, ni0, nj0);
            nai = sp[ni0 * kRepBlock + lane];
            naj = sp[nj0 * kRepBlock + lane];
        }
        // ---- partials to every CTA, one cluster barrier
        float4* buf = cred + (size_t)(m & 1) * CW * kRepBlock;
        const float4 mine = make_float4(h[0], h[1], h[2], h[3]);
        for (int q = 0; q < C; q++) st_cluster_f4(buf + gw * kRepBlock + lane, (uint32_t)q, mine);
        // a warp that aborts raises the flag in every CTA before the barrier,
        // so all of them read it after the same barrier and leave together
        if (!ok && lane == 0)
            for (int q = 0; q < C; q++) st_cluster_u32(cflag, (uint32_t)q, 1u);
        cluster_sync();
        if (*(volatile int*)cflag) {
            aborted = true;
            break;
        }

        // ---- decision m, the same in every warp
        const float4 hs = sum_partials(buf + lane, C, W, kRepBlock);
        const float dix = cain.x - cai.x, diy = cain.y - cai.y;
        const float djx = cajn.x - caj.x, djy = cajn.y - caj.y;
        const float dE = -fmaf(dix, hs.x, -diy * hs.y) - fmaf(djx, hs.z, -djy * hs.w);
        // mc.cu:288-297: beta == 0 accepts everything; otherwise dE <= 0 or u < exp(-beta dE)
        bool accept;
        if (beta_d == 0.0) accept = true;
        else accept = (dE <= 0.f) || (cu < expf(-beta * dE));
        const float2 ai_post = accept ? cain : cai, aj_post = accept ? cajn : caj;
        if (warp == 0) {
            if (accept) {
                E += (double)dE;
                nacc++;
            }
            nprop++;
            if (writer && P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + lane == P.trace_rep &&
                active) {
                const long long sw = sweep0 + m / steps;
                const long long idx = (sw - P.trace_sweep0) * steps + m % steps;
                if (idx >= 0 && idx < P.trace_cap) {
                    pspin_move_record* rec = reinterpret_cast<pspin_move_record*>(P.trace) + idx;
                    rec->i0 = ci0; rec->j0 = cj0;
                    rec->ai_old[0] = cai.x; rec->ai_old[1] = cai.y;
                    rec->aj_old[0] = caj.x; rec->aj_old[1] = caj.y;
                    rec->ai_new[0] = cain.x; rec->ai_new[1] = cain.y;
                    rec->aj_new[0] = cajn.x; rec->aj_new[1] = cajn.y;
                    rec->dE = dE;
                    rec->accepted = accept ? 1 : 0;
                    rec->log_q_ratio = 0.f;
                    rec->log_u = logf(cu);
                }
            }
        }
        // ---- proposal m+1 and the final values of the state it reads
        if (m + 1 < total) {
            const float2 ai1 = ni0 == ci0 ? ai_post : (ni0 == cj0 ? aj_post : nai);
            const float2 aj1 = nj0 == ci0 ? ai_post : (nj0 == cj0 ? aj_post : naj);
            const int pi0 = ci0, pj0 = cj0;
            ci0 = ni0;
            cj0 = nj0;
            take_pre(m + 1, ai1, aj1);
            sp[pi0 * kRepBlock + lane] = pi0 == cj0 ? cajn : ai_post;
            sp[pj0 * kRepBlock + lane] = pj0 == cj0 ? cajn : aj_post;
            sp[cj0 * kRepBlock + lane] = cajn;     // h_i of move m+1 is evaluated at its proposed a_j
        } else {
            sp[ci0 * kRepBlock + lane] = ai_post;
            sp[cj0 * kRepBlock + lane] = aj_post;
        }
    }
    if (aborted) drain_ring(bars, kStages, consumed, issued, P.status);   // state stays as before the launch
    __syncthreads();                           // every warp's final writes before the write-back
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
    cluster_sync();                            // no CTA leaves while a remote store may target it
}

template <int VARIANT, bool kBatch>
static cudaError_t launch_one(const SweepParams& p, int n_units, size_t smem, cudaStream_t st, bool check_only,
                              int* max_clusters) {
    auto kern = sweep_cluster_kernel<VARIANT, kBatch>;
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
    cfg.numAttrs = 1;
    if (check_only) return cudaOccupancyMaxActiveClusters(max_clusters, kern, &cfg);
    e = cudaLaunchKernelEx(&cfg, kern, p);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// max_clusters != null: only reports how many clusters of this shape can be
// resident (0: the shape does not fit)
cudaError_t launch_sweep_cluster(const SweepParams& p, int n_units, int variant, int max_N, cudaStream_t st,
                                 int* max_clusters) {
    if (n_units <= 0) return cudaSuccess;
    if (p.cluster < 2 || p.cluster > 16 || (kSplit % (p.cluster * p.warps)) != 0) return cudaErrorInvalidValue;
    const size_t smem = cluster_smem_bytes(max_N, p.warps, p.cluster);
    const bool check = max_clusters != nullptr;
    int sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    // batched record loads when the launch leaves SMs without a CTA
    const bool batch = (long long)n_units * p.cluster <= sms;
    if (variant == 0)
        return batch ? launch_one<0, true>(p, n_units, smem, st, check, max_clusters)
                     : launch_one<0, false>(p, n_units, smem, st, check, max_clusters);
    return batch ? launch_one<1, true>(p, n_units, smem, st, check, max_clusters)
                 : launch_one<1, false>(p, n_units, smem, st, check, max_clusters);
}

size_t cluster_smem_bytes_host(int N, int warps, int C) { return cluster_smem_bytes(N, warps, C); }

}  // namespace pspin
