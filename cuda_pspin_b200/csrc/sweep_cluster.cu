// sweep_cluster.cu -- the plain pair-rotation sweep with one replica block
// split over a thread-block cluster of C CTAs (C = 2..16), for workloads
// with fewer replica blocks than SMs (one large sample, few replicas).
//
// Same moves, RNG streams and Metropolis rule as sweep_kernel.  Every CTA of
// the cluster holds the block's amplitudes in its own shared memory and
// reads 1/C of every site list through its own TMA rings.  Per move:
//   1. each CTA sums its warps' partial fields and stores the float4 of
//      every lane into slot [rank] of every CTA's exchange buffer
//      (distributed shared memory, mapa + st.shared::cluster);
//   2. one cluster barrier (release / acquire);
//   3. warp 0 of every CTA adds the C partials in rank order -- the same
//      numbers in the same order everywhere -- and takes the same Metropolis
//      decision on the same random words, so the CTAs' amplitude copies stay
//      identical without broadcasting them.
// The exchange buffer is double-buffered by move parity: a CTA can be at
// most one move ahead of another (it cannot pass the next cluster barrier
// before the slower CTA has read the current buffer).  Rank 0 writes the
// results back.
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

// the exchange buffer follows the plain kernel's layout, rounded up to 16
// bytes (float4 stores and loads; with one warp that layout ends at 8 mod 16)
__host__ __device__ inline size_t cluster_buffer_offset(int N, int warps) {
    return (sweep_smem_bytes(N, warps) + 15) & ~(size_t)15;
}

// exchange buffer [2][C][32] float4, then the cluster's abort flag (one word)
inline size_t cluster_smem_bytes(int N, int warps, int C) {
    return cluster_buffer_offset(N, warps) + (size_t)2 * C * kRepBlock * sizeof(float4) + 16;
}

template <int VARIANT>
__global__ void __launch_bounds__(256, 2) sweep_cluster_kernel(const SweepParams P) {
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
    float2* sp = reinterpret_cast<float2*>(smem_raw);                          // [(N+1)][32]
    float4* red = reinterpret_cast<float4*>(sp + (size_t)(N + 1) * kRepBlock);  // [W][32]
    int2* ring_all = reinterpret_cast<int2*>(red + (size_t)W * kRepBlock);
    int2* ring = ring_all + (size_t)warp * kStages * kStage;
    uint64_t* bars_all = reinterpret_cast<uint64_t*>(ring_all + (size_t)W * kStages * kStage);
    uint64_t* bars = bars_all + warp * kStages;
    float4* cred = reinterpret_cast<float4*>(smem_raw + cluster_buffer_offset(N, W));   // [2][C][32]
    // raised in every CTA of the cluster by a CTA that aborts (see below)
    int* cflag = reinterpret_cast<int*>(cred + (size_t)2 * C * kRepBlock);

    const bool active = lane < U.rep_count;
    const bool writer = rank == 0;
    const int64_t gr = S.rep_off + U.rep_begin + lane;

    for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
        const int site = idx >> 5, l = idx & 31;
        float2 v = make_float2(1.f, 0.f);
        if (l < U.rep_count) v = P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l];
        sp[idx] = v;
    }
    if (threadIdx.x < kRepBlock) sp[N * kRepBlock + threadIdx.x] = make_float2(1.f, 0.f);  // virtual site
    if (threadIdx.x == 0) *cflag = 0;

    double E = 0.0, beta_d = 0.0;
    float beta = 0.f;
    long long nacc = 0, nprop = 0;
    uint32_t k0 = 0, k1 = 0;
    if (warp == 0 && active) {
        E = P.energy[gr];
        beta_d = P.beta[gr];
        beta = (float)beta_d;
        const uint64_t key = P.key[gr];
        k0 = (uint32_t)key;
        k1 = (uint32_t)(key >> 32);
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2;
    const int total = P.nsweeps * steps;
    const int TW = C * W, gw = (int)rank * W + warp;

    Stream<2, false> st;
    st.key0 = S.pair_key0;
    st.key1 = S.pair_key1;
    st.N = N;
    st.site_chunks = P.site_chunks + S.split_off;
    st.pair_chunks = nullptr;
    st.sweep0 = sweep0;
    st.steps = steps;
    st.total = total;
    st.part0 = gw * (kSplit / TW);
    st.part1 = (gw + 1) * (kSplit / TW);

    if (lane == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(bars + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_shared();
    }
    __syncwarp();
    Cursor pc = st.first();
    uint32_t issued = 0, consumed = 0;
    bool ok = true;
    auto issue = [&]() {
        if (pc.m >= total) return;
        const uint32_t slot = issued % kStages;
        if (lane == 0) {
            const int64_t b = __ldg(P.chunk_start + pc.c), e = __ldg(P.chunk_start + pc.c + 1);
            const uint32_t bytes = (uint32_t)((e - b) * sizeof(int2));
            mbar_expect_tx(bars + slot, bytes);
            bulk_g2s(ring + slot * kStage, P.entries + b, bytes, bars + slot);
        }
        issued++;
        st.next(pc);
    };
    for (int s = 0; s < kStages; s++) issue();

    int ci0 = 0, cj0 = 0;
    float2 cai = make_float2(0.f, 0.f), caj = cai, cain = cai, cajn = cai;
    float cu = 0.f;
    auto prepare = [&](int m) {
        const long long sw = sweep0 + m / steps;
        const int k = m % steps;
        pair_pick(S.pair_key0, S.pair_key1, (uint64_t)sw, (uint32_t)k, N, ci0, cj0);
        cai = sp[ci0 * kRepBlock + lane];
        caj = sp[cj0 * kRepBlock + lane];
        const U4 w = move_words(k0, k1, (uint64_t)sw, (uint32_t)k);
        propose<VARIANT>(cai, caj, w, cain, cajn);
        cu = u01f(w.w);
        sp[cj0 * kRepBlock + lane] = cajn;     // h_i is evaluated at the proposed a_j
    };

    __shared__ __align__(8) uint64_t stall_bar;      // test hook: nothing arrives on it
    if (threadIdx.x == 0 && P.stall_move >= 0) {
        mbar_init(&stall_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == 0 && total > 0) prepare(0);
    __syncthreads();
    cluster_sync();                            // every CTA runs before the first remote store

    bool aborted = false;
    for (int m = 0; m < total; m++) {
        const long long sw = sweep0 + m / steps;
        const int k = m % steps;
        float h[4] = {0.f, 0.f, 0.f, 0.f};
        if (m == P.stall_move) ok = stall_wait(&stall_bar, P.status, P.wait_clocks);
        for (int which = 0; which < 2 && ok; which++) {
            int c, c_end;
            st.range(m, which, c, c_end);
            for (; c < c_end; c++) {
                const uint32_t slot = consumed % kStages;
                ok = ring_wait(bars + slot, (consumed / kStages) & 1u, P.status, P.wait_clocks);
                if (!ok) break;                    // stop consuming and issuing; abort below
                const int n = (int)(__ldg(P.chunk_start + c + 1) - __ldg(P.chunk_start + c));
                if (S.fc_tiles) accumulate_tiles(ring + slot * kStage, n, sp, lane, h[2 * which], h[2 * which + 1]);
                else accumulate_chunk(ring + slot * kStage, n, sp, lane, h[2 * which], h[2 * which + 1]);
                consumed++;
                __syncwarp();
                if (lane == 0) fence_async_shared();
                issue();
            }
        }
        red[warp * kRepBlock + lane] = make_float4(h[0], h[1], h[2], h[3]);
        const bool bad = __syncthreads_or(!ok);
        float4* buf = cred + (size_t)(m & 1) * C * kRepBlock;
        if (warp == 0) {
            float4 hs = red[lane];
            for (int w = 1; w < W; w++) {
                const float4 v = red[w * kRepBlock + lane];
                hs.x += v.x; hs.y += v.y; hs.z += v.z; hs.w += v.w;
            }
            for (int q = 0; q < C; q++) st_cluster_f4(buf + rank * kRepBlock + lane, (uint32_t)q, hs);
            // an aborting CTA raises the flag in every CTA before the barrier,
            // so all of them read it after the same barrier and leave together
            if (bad && lane == 0)
                for (int q = 0; q < C; q++) st_cluster_u32(cflag, (uint32_t)q, 1u);
        }
        cluster_sync();
        if (*(volatile int*)cflag) {
            aborted = true;
            break;
        }

        if (warp == 0) {
            float4 hs = buf[lane];
            for (int q = 1; q < C; q++) {
                const float4 v = buf[q * kRepBlock + lane];
                hs.x += v.x; hs.y += v.y; hs.z += v.z; hs.w += v.w;
            }
            const float dix = cain.x - cai.x, diy = cain.y - cai.y;
            const float djx = cajn.x - caj.x, djy = cajn.y - caj.y;
            const float dE = -fmaf(dix, hs.x, -diy * hs.y) - fmaf(djx, hs.z, -djy * hs.w);
            bool accept;
            if (beta_d == 0.0) accept = true;
            else accept = (dE <= 0.f) || (cu < expf(-beta * dE));
            if (accept) {
                sp[ci0 * kRepBlock + lane] = cain;
                E += (double)dE;
                nacc++;
            } else {
                sp[cj0 * kRepBlock + lane] = caj;
            }
            nprop++;
            if (writer && P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + lane == P.trace_rep &&
                active) {
                const long long idx = (sw - P.trace_sweep0) * steps + k;
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
            if (m + 1 < total) prepare(m + 1);
        }
        __syncthreads();
    }
    if (aborted) drain_ring(bars, kStages, consumed, issued, P.status);   // state stays as before the launch
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

template <int VARIANT>
static cudaError_t launch_one(const SweepParams& p, int n_units, size_t smem, cudaStream_t st, bool check_only,
                              int* max_clusters) {
    auto kern = sweep_cluster_kernel<VARIANT>;
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
    return variant == 0 ? launch_one<0>(p, n_units, smem, st, check, max_clusters)
                        : launch_one<1>(p, n_units, smem, st, check, max_clusters);
}

size_t cluster_smem_bytes_host(int N, int warps, int C) { return cluster_smem_bytes(N, warps, C); }

}  // namespace pspin
