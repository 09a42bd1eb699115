// sweep.cu -- the pair-rotation Metropolis sweep (dense sphere and sparse
// cube), hand-written for sm_100a.
//
// Replaces mc_sweep_kernel (mc.cu:66-318) and mc_sparse_sweep_kernel
// (mc_sparse.cu:63-253).  Same move set, same Metropolis rule; different
// organisation:
//
//  * One CTA = one unit = up to 32 replicas of one sample; lane l of every
//    warp owns replica rep_begin+l.  All replicas of a sample propose on the
//    same pair at the same step (the pair stream belongs to the sample, not
//    to the replica), so each coupling entry is read once per warp and used
//    by 32 replicas.  Pair choice does not depend on the state, so every
//    replica still runs a random-scan Metropolis chain with the reference's
//    stationary law.
//  * dE from local fields.  E is affine in a_i for fixed other sites, so
//      E(a_i',a_j') - E(a_i,a_j) = -Re[da_i h_i(a_j')] - Re[da_j h_j(a_i)]
//    exactly, where h_i(a_j') is site i's field evaluated with the proposed
//    a_j.  Warp 0 writes the proposed a_j into j's shared-memory slot before
//    the fields are accumulated and restores it on rejection: no
//    quartet-by-quartet old/new products and no separate pair term.
//  * Fields are accumulated from per-site lists grouped by (partner, first
//    opposite site): per data entry one shared-memory gather and two FFMA.
//    The W warps of a CTA split both lists; partial fields meet in shared
//    memory and warp 0 takes the Metropolis decisions.
//  * The lists reach shared memory through per-warp TMA (cp.async.bulk)
//    rings that prefetch across moves, so no warp waits on L2 latency.
//  * FP32 amplitudes and fields; the running energy is FP64.
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

template <int VARIANT>
__global__ void __launch_bounds__(256, 3) sweep_kernel(const SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Unit U = P.units[blockIdx.x];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N;
    const int R = S.R;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int W = P.warps;
    float2* sp = reinterpret_cast<float2*>(smem_raw);                          // [(N+1)][32]
    float4* red = reinterpret_cast<float4*>(sp + (size_t)(N + 1) * kRepBlock);  // [W][32]
    int2* ring = reinterpret_cast<int2*>(red + (size_t)W * kRepBlock) + (size_t)warp * kStages * kStage;
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<int2*>(red + (size_t)W * kRepBlock) +
                                                 (size_t)W * kStages * kStage) + warp * kStages;

    const bool active = lane < U.rep_count;
    const int64_t gr = S.rep_off + U.rep_begin + lane;

    load_block_amplitudes(sp, P.spins + S.spin_off + U.rep_begin, R, N, kRepBlock, U.rep_count);
    if (threadIdx.x < kRepBlock) sp[N * kRepBlock + threadIdx.x] = make_float2(1.f, 0.f);  // virtual site

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

    Stream<2> st;
    st.key0 = S.pair_key0;
    st.key1 = S.pair_key1;
    st.N = N;
    st.site_chunks = P.site_chunks + S.split_off;
    st.pair_chunks = nullptr;
    st.sweep0 = sweep0;
    st.steps = steps;
    st.total = total;
    st.part0 = warp * (kSplit / W);
    st.part1 = (warp + 1) * (kSplit / W);

    // ring set-up and prologue: kStages chunks in flight
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

    // warp-0 registers describing the pending move
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
                else accumulate_records_1(ring + slot * kStage, n, sp, lane, h[2 * which], h[2 * which + 1]);
                consumed++;
                __syncwarp();
                if (lane == 0) fence_async_shared();
                issue();
            }
        }
        red[warp * kRepBlock + lane] = make_float4(h[0], h[1], h[2], h[3]);
        if (__syncthreads_or(!ok)) {              // CTA-uniform: every warp leaves at this move
            aborted = true;
            break;
        }

        if (warp == 0) {
            float4 hs = red[lane];
            for (int w = 1; w < W; w++) {
                const float4 v = red[w * kRepBlock + lane];
                hs.x += v.x; hs.y += v.y; hs.z += v.z; hs.w += v.w;
            }
            const float dix = cain.x - cai.x, diy = cain.y - cai.y;
            const float djx = cajn.x - caj.x, djy = cajn.y - caj.y;
            const float dE = -fmaf(dix, hs.x, -diy * hs.y) - fmaf(djx, hs.z, -djy * hs.w);
            // mc.cu:288-297: beta == 0 accepts everything; otherwise dE <= 0
            // or u < exp(-beta dE)
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
            if (P.trace != nullptr && U.sample == P.trace_sample &&
                U.rep_begin + lane == P.trace_rep && active) {
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
    if (aborted) {
        // copies still in flight: wait for them (bounded); the replicas keep
        // their state from before the launch
        drain_ring(bars, kStages, consumed, issued, P.status);
        return;
    }

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

cudaError_t launch_sweep(const SweepParams& p, int n_units, int variant, int max_N, cudaStream_t st) {
    if (n_units <= 0) return cudaSuccess;
    const size_t smem = sweep_smem_bytes(max_N, p.warps);
    const dim3 block(32 * p.warps);
    if (variant == 0) {
        cudaError_t e = cudaFuncSetAttribute(sweep_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        sweep_kernel<0><<<n_units, block, smem, st>>>(p);
    } else {
        cudaError_t e = cudaFuncSetAttribute(sweep_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        sweep_kernel<1><<<n_units, block, smem, st>>>(p);
    }
    return cudaGetLastError();
}

}  // namespace pspin
