// sweep_resident.cu -- the plain pair-rotation sweep for samples whose whole
// set of site lists fits in shared memory next to the amplitudes (sparse
// samples: ~8 list entries per site).
//
// Same moves, RNG streams and Metropolis rule as sweep_kernel.  The lists
// are copied into shared memory once per launch, so a move reads them
// without TMA copies; site m's list is the contiguous range of its chunks
// (groups or tiles never span chunks; the padding entry of an odd chunk is
// an empty group).
//
// Concurrent commuting moves.  With K warps per replica block, the moves
// are taken in windows of 32: the lanes of warp 0 draw the window's pair
// picks (one Philox call each), every warp precomputes the random words,
// sines and cosines of its share of the window's proposals, and the warps
// mark, for every move, the earlier moves of the window it does not commute
// with -- move b does not commute with
// move a when one of b's sites is a site of a or shares a quartet (or a g2
// term) with one: then b's proposal or fields would read an amplitude that a
// changes.  The window is cut greedily, in move order, into batches of at
// most K moves that pairwise commute, and the warps run the moves of a batch
// at once, warp w the batch's w-th move, each for the block's 32 replicas.
// Moves that commute give the same result in either order (the same fields,
// proposals and decisions on the same random words), so a batch equals the
// same moves run one after another, and the chain is the one-warp chain
// bit for bit: the running energy adds the moves' dE in move order.  One CTA
// barrier per batch.  At N=512 with N selected quartets a batch holds ~3.9
// moves with K=8.
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

// Shared memory: amplitudes [(N+1)][32] float2 ((N+1)*256 bytes, so the list
// entries that follow are 16-byte aligned: tiles are read as int4), the
// sample's list entries, site ranges [N] int2, the window's pair picks and
// (sweep, step) of each move [32] int2 each, batch bounds [34] int,
// conflict masks [32] u32, per-batch dE and decisions [2][K][32] (float,
// int), the window's precomputed proposal parts [32 moves][7][32] float,
// and (K > 1) the neighbour-mask rows of the window's pairs [32][2][ceil(N/32)].
inline size_t resident_smem_bytes(int N, int64_t entries, int K) {
    size_t b = (size_t)(N + 1) * kRepBlock * sizeof(float2) + (size_t)entries * sizeof(int2) +
               (size_t)N * sizeof(int2) + 2 * 32 * sizeof(int2) + 34 * sizeof(int) + 32 * sizeof(uint32_t) +
               (size_t)2 * K * kRepBlock * (sizeof(float) + sizeof(int)) + (size_t)32 * 7 * kRepBlock * sizeof(float);
    if (K > 1) b += (size_t)64 * ((N + 31) / 32) * sizeof(uint32_t);
    return b;
}

template <int VARIANT>
__global__ void __launch_bounds__(256) sweep_resident_kernel(const SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Unit U = P.units[blockIdx.x];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N, R = S.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int K = (int)(blockDim.x >> 5);
    const int owner = K - 1;                   // keeps the running energy and counters
    const int wpr = (N + 31) >> 5;             // words per neighbour-mask row
    const uint32_t* nbm = P.nbmask + S.nb_off; // read through L1
    const int* sc = P.site_chunks + S.split_off;
    const int64_t e0 = __ldg(P.chunk_start + __ldg(sc));
    const int64_t e1 = __ldg(P.chunk_start + __ldg(sc + (int64_t)(N - 1) * (kSplit + 1) + kSplit));
    float2* sp = reinterpret_cast<float2*>(smem_raw);
    int2* L = reinterpret_cast<int2*>(sp + (size_t)(N + 1) * kRepBlock);
    int2* rng_site = L + (e1 - e0);
    int2* picks = rng_site + N;
    int2* mk = picks + 32;                                     // (sweep - sweep0, step) of each move
    int* bounds = reinterpret_cast<int*>(mk + 32);             // [0..32] batch starts, [33] batch count
    uint32_t* cm = reinterpret_cast<uint32_t*>(bounds + 34);   // [32]
    float* dEx = reinterpret_cast<float*>(cm + 32);            // [2][K][32]
    int* acx = reinterpret_cast<int*>(dEx + 2 * K * kRepBlock);  // [2][K][32]
    float* tr = reinterpret_cast<float*>(acx + 2 * K * kRepBlock);  // [32][7][32]
    uint32_t* nrow = reinterpret_cast<uint32_t*>(tr + 32 * 7 * kRepBlock);   // [32][2][wpr]
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        const int64_t b = __ldg(P.chunk_start + __ldg(sc + (int64_t)m * (kSplit + 1)));
        const int64_t e = __ldg(P.chunk_start + __ldg(sc + (int64_t)m * (kSplit + 1) + kSplit));
        rng_site[m] = make_int2((int)(b - e0), (int)(e - e0));
    }
    load_block_range(L, P.entries + e0, e1 - e0);
    load_block_amplitudes(sp, P.spins + S.spin_off + U.rep_begin, R, N, kRepBlock, U.rep_count);
    if (threadIdx.x < kRepBlock) sp[N * kRepBlock + threadIdx.x] = make_float2(1.f, 0.f);   // virtual site

    const bool active = lane < U.rep_count;
    const int64_t gr = S.rep_off + U.rep_begin + lane;
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
        if (warp == owner) E = P.energy[gr];
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2, total = P.nsweeps * steps;
    // is `site` a site of the window's move j or a neighbour of one?
    auto in_reach = [&](int site, int j) {
        const int2 q = picks[j];
        const uint32_t* rows = nrow + 2 * j * wpr;
        return site == q.x || site == q.y || (((rows[site >> 5] | rows[wpr + (site >> 5)]) >> (site & 31)) & 1u);
    };
    // the owner warp's running energy and counters take a batch's moves in move order
    auto account = [&](int par, int n) {
        for (int w = 0; w < n; w++) {
            if (acx[(par * K + w) * kRepBlock + lane]) {
                E += (double)dEx[(par * K + w) * kRepBlock + lane];
                nacc++;
            }
            nprop++;
        }
    };
    __syncthreads();

    long long batches = 0;
    int prev = 0;                              // moves in the previous batch
    for (int m0 = 0; m0 < total; m0 += 32) {
        const int n = min(32, total - m0);
        if (warp == 0) {                       // the window's pairs
            int i0 = 0, j0 = 1, sw = 0, kk = 0;
            if (lane < n) {
                sw = (m0 + lane) / steps;
                kk = (m0 + lane) % steps;
                pair_pick(S.pair_key0, S.pair_key1, (uint64_t)(sweep0 + sw), (uint32_t)kk, N, i0, j0);
            }
            picks[lane] = make_int2(i0, j0);
            mk[lane] = make_int2(sw, kk);
            cm[lane] = 0u;
        }
        // every warp: the state-independent parts of the proposals of its share
        // of the window's moves (random words, sines and cosines), for its lanes
        for (int t = warp; t < n; t += K) {
            const int m = m0 + t;
            float tt[7];
            move_trig<VARIANT>(move_words(k0, k1, (uint64_t)(sweep0 + m / steps), (uint32_t)(m % steps)), tt);
#pragma unroll
            for (int q = 0; q < 7; q++) tr[(t * 7 + q) * kRepBlock + lane] = tt[q];
        }
        __syncthreads();
        if (K > 1) {
            // the neighbour-mask rows of the window's sites, all loads in flight at once
            const int tot = n * 2 * wpr;
            for (int i0 = threadIdx.x; i0 < tot; i0 += kInFlight * blockDim.x) {
                uint32_t v[kInFlight];
#pragma unroll
                for (int u = 0; u < kInFlight; u++) {
                    const int idx = i0 + u * (int)blockDim.x;
                    v[u] = 0u;
                    if (idx < tot) {
                        const int j = idx / (2 * wpr), r = idx - j * 2 * wpr;
                        const int2 q = picks[j];
                        v[u] = __ldg(nbm + (r < wpr ? q.x * wpr + r : q.y * wpr + (r - wpr)));
                    }
                }
#pragma unroll
                for (int u = 0; u < kInFlight; u++) {
                    const int idx = i0 + u * (int)blockDim.x;
                    if (idx < tot) nrow[idx] = v[u];
                }
            }
            __syncthreads();
            // conflict masks: the earlier moves of the window that move `lane`
            // does not commute with, the earlier moves shared out over the warps
            uint32_t part = 0;
            if (lane < n) {
                const int2 me = picks[lane];
                for (int j = warp; j < lane; j += K)
                    if (in_reach(me.x, j) || in_reach(me.y, j)) part |= 1u << j;
            }
            if (part) atomicOr(cm + lane, part);
            __syncthreads();
            if (warp == 0) {
                // greedy cut in move order: a batch [s0, e) ends at the first move
                // that does not commute with one of [s0, itself), or after K moves
                const uint32_t mask = cm[lane];
                int nb = 0;
                for (int s0 = 0; s0 < n;) {
                    const unsigned bad = __ballot_sync(0xffffffffu, lane > s0 && lane < n && (mask >> s0) != 0u);
                    const int e = min(bad ? __ffs(bad) - 1 : n, min(n, s0 + K));
                    if (lane == 0) bounds[nb] = s0;
                    nb++;
                    s0 = e;
                }
                if (lane == 0) {
                    bounds[nb] = n;
                    bounds[33] = nb;
                }
            }
            __syncthreads();
        } else {
            if (lane == 0) {
                for (int b = 0; b <= n; b++) bounds[b] = b;
                bounds[33] = n;
            }
            __syncwarp();
        }
        const int nb = bounds[33];
        for (int b = 0; b < nb; b++) {
            const int bs = bounds[b], be = bounds[b + 1];
            const int par = (int)(batches & 1);
            if (warp == owner && batches > 0) account(par ^ 1, prev);
            if (warp < be - bs) {
                const int t = bs + warp;
                const int2 pq = picks[t], swk = mk[t];
                const int i0 = pq.x, j0 = pq.y;
                float tt[7];
#pragma unroll
                for (int q = 0; q < 7; q++) tt[q] = tr[(t * 7 + q) * kRepBlock + lane];
                const float2 ai = sp[i0 * kRepBlock + lane], aj = sp[j0 * kRepBlock + lane];
                float2 ain, ajn;
                propose_with<VARIANT>(ai, aj, tt, ain, ajn);
                const float cu = tt[6];
                sp[j0 * kRepBlock + lane] = ajn;       // h_i is evaluated at the proposed a_j
                __syncwarp();
                float hix = 0.f, hiy = 0.f, hjx = 0.f, hjy = 0.f;
                const int2 ri = rng_site[i0], rj = rng_site[j0];
                if (S.fc_tiles) {
                    accumulate_tiles(L + ri.x, ri.y - ri.x, sp, lane, hix, hiy);
                    accumulate_tiles(L + rj.x, rj.y - rj.x, sp, lane, hjx, hjy);
                } else if (S.single_groups) {
                    accumulate_records<4, true>(L + ri.x, ri.y - ri.x, sp, lane, hix, hiy);
                    accumulate_records<4, true>(L + rj.x, rj.y - rj.x, sp, lane, hjx, hjy);
                } else {
                    accumulate_records(L + ri.x, ri.y - ri.x, sp, lane, hix, hiy);
                    accumulate_records(L + rj.x, rj.y - rj.x, sp, lane, hjx, hjy);
                }
                const float dix = ain.x - ai.x, diy = ain.y - ai.y;
                const float djx = ajn.x - aj.x, djy = ajn.y - aj.y;
                const float dE = -fmaf(dix, hix, -diy * hiy) - fmaf(djx, hjx, -djy * hjy);
                bool accept;
                if (beta_d == 0.0) accept = true;
                else accept = (dE <= 0.f) || (cu < expf(-beta * dE));
                __syncwarp();
                if (accept) sp[i0 * kRepBlock + lane] = ain;
                else sp[j0 * kRepBlock + lane] = aj;
                dEx[(par * K + warp) * kRepBlock + lane] = dE;
                acx[(par * K + warp) * kRepBlock + lane] = accept ? 1 : 0;
                if (P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + lane == P.trace_rep && active) {
                    const long long idx = (long long)swk.x * steps + swk.y + (sweep0 - P.trace_sweep0) * steps;
                    if (idx >= 0 && idx < P.trace_cap) {
                        pspin_move_record* rec = reinterpret_cast<pspin_move_record*>(P.trace) + idx;
                        rec->i0 = i0; rec->j0 = j0;
                        rec->ai_old[0] = ai.x; rec->ai_old[1] = ai.y;
                        rec->aj_old[0] = aj.x; rec->aj_old[1] = aj.y;
                        rec->ai_new[0] = ain.x; rec->ai_new[1] = ain.y;
                        rec->aj_new[0] = ajn.x; rec->aj_new[1] = ajn.y;
                        rec->dE = dE;
                        rec->accepted = accept ? 1 : 0;
                        rec->log_q_ratio = 0.f;
                        rec->log_u = logf(cu);
                    }
                }
            }
            __syncthreads();
            prev = be - bs;
            batches++;
        }
    }
    if (warp == owner && batches > 0) account((int)((batches - 1) & 1), prev);
    for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
        const int site = idx >> 5, l = idx & 31;
        if (l < U.rep_count) P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l] = sp[idx];
    }
    if (warp == owner && active) {
        P.energy[gr] = E;
        P.accepted[gr] += nacc;
        P.proposed[gr] += nprop;
    }
}

size_t resident_smem_bytes_host(int N, int64_t entries, int warps) { return resident_smem_bytes(N, entries, warps); }

cudaError_t launch_sweep_resident(const SweepParams& p, int n_units, int variant, int max_N, int64_t max_entries,
                                  cudaStream_t st) {
    if (n_units <= 0) return cudaSuccess;
    if (p.warps < 1 || p.warps > 8) return cudaErrorInvalidValue;
    const size_t smem = resident_smem_bytes(max_N, max_entries, p.warps);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    auto kern = variant == 0 ? sweep_resident_kernel<0> : sweep_resident_kernel<1>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<n_units, 32 * p.warps, smem, st>>>(p);
    return cudaGetLastError();
}

}  // namespace pspin
