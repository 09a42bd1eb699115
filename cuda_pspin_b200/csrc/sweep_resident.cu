// sweep_resident.cu -- the plain pair-rotation sweep for samples whose whole
// set of site lists fits in shared memory next to the amplitudes (sparse
// samples: ~8 list entries per site), one warp per replica block.
//
// Same moves, RNG streams and Metropolis rule as sweep_kernel.  The lists
// are copied into shared memory once per launch, so a move reads them
// without TMA copies or barriers; the 32 lanes evaluate the pair picks of
// the next 32 moves with one Philox call each; every move runs
// warp-synchronously (no CTA barrier).  Site m's list is the contiguous
// range of its chunks (groups or tiles never span chunks; the padding entry
// of an odd chunk is an empty group).
#include "sweep_common.cuh"
#include "../../include/pspin.h"

namespace pspin {

// amplitudes [(N+1)][32] float2 ((N+1)*256 bytes), the sample's list entries
// (16-byte aligned there: tiles are read as int4), site ranges [N] int2,
// pair picks [32] int2
inline size_t resident_smem_bytes(int N, int64_t entries) {
    return (size_t)(N + 1) * kRepBlock * sizeof(float2) + (size_t)entries * sizeof(int2) + (size_t)N * sizeof(int2) +
           32 * sizeof(int2);
}

template <int VARIANT>
__global__ void __launch_bounds__(32) sweep_resident_kernel(const SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Unit U = P.units[blockIdx.x];
    const SampleDev S = P.samples[U.sample];
    const int N = S.N, R = S.R;
    const int lane = threadIdx.x;
    const int* sc = P.site_chunks + S.split_off;
    const int64_t e0 = __ldg(P.chunk_start + __ldg(sc));
    const int64_t e1 = __ldg(P.chunk_start + __ldg(sc + (int64_t)(N - 1) * (kSplit + 1) + kSplit));
    float2* sp = reinterpret_cast<float2*>(smem_raw);
    int2* L = reinterpret_cast<int2*>(sp + (size_t)(N + 1) * kRepBlock);
    int2* rng_site = L + (e1 - e0);
    int2* picks = rng_site + N;
    for (int m = lane; m < N; m += 32) {
        const int64_t b = __ldg(P.chunk_start + __ldg(sc + (int64_t)m * (kSplit + 1)));
        const int64_t e = __ldg(P.chunk_start + __ldg(sc + (int64_t)m * (kSplit + 1) + kSplit));
        rng_site[m] = make_int2((int)(b - e0), (int)(e - e0));
    }
    for (int64_t t = lane; t < e1 - e0; t += 32) L[t] = P.entries[e0 + t];
    for (int idx = lane; idx < N * kRepBlock; idx += 32) {
        const int site = idx >> 5, l = idx & 31;
        float2 v = make_float2(1.f, 0.f);
        if (l < U.rep_count) v = P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l];
        sp[idx] = v;
    }
    sp[N * kRepBlock + lane] = make_float2(1.f, 0.f);     // virtual site

    const bool active = lane < U.rep_count;
    const int64_t gr = S.rep_off + U.rep_begin + lane;
    double E = 0.0, beta_d = 0.0;
    float beta = 0.f;
    long long nacc = 0, nprop = 0;
    uint32_t k0 = 0, k1 = 0;
    if (active) {
        E = P.energy[gr];
        beta_d = P.beta[gr];
        beta = (float)beta_d;
        const uint64_t key = P.key[gr];
        k0 = (uint32_t)key;
        k1 = (uint32_t)(key >> 32);
    }
    const long long sweep0 = *P.sweep_counter;
    const int steps = N / 2, total = P.nsweeps * steps;
    __syncwarp();

    for (int m = 0; m < total; m++) {
        if ((m & 31) == 0) {                   // pair picks of moves m .. m+31, one per lane
            const int mm = m + lane;
            int i0 = 0, j0 = 1;
            if (mm < total)
                pair_pick(S.pair_key0, S.pair_key1, (uint64_t)(sweep0 + mm / steps), (uint32_t)(mm % steps), N, i0, j0);
            picks[lane] = make_int2(i0, j0);
            __syncwarp();
        }
        const long long sw = sweep0 + m / steps;
        const int k = m % steps;
        const int2 pq = picks[m & 31];
        const int i0 = pq.x, j0 = pq.y;
        const U4 w = move_words(k0, k1, (uint64_t)sw, (uint32_t)k);
        const float2 ai = sp[i0 * kRepBlock + lane], aj = sp[j0 * kRepBlock + lane];
        float2 ain, ajn;
        propose<VARIANT>(ai, aj, w, ain, ajn);
        const float cu = u01f(w.w);
        sp[j0 * kRepBlock + lane] = ajn;       // h_i is evaluated at the proposed a_j
        __syncwarp();
        float hix = 0.f, hiy = 0.f, hjx = 0.f, hjy = 0.f;
        const int2 ri = rng_site[i0], rj = rng_site[j0];
        if (S.fc_tiles) {
            accumulate_tiles(L + ri.x, ri.y - ri.x, sp, lane, hix, hiy);
            accumulate_tiles(L + rj.x, rj.y - rj.x, sp, lane, hjx, hjy);
        } else {
            accumulate_chunk(L + ri.x, ri.y - ri.x, sp, lane, hix, hiy);
            accumulate_chunk(L + rj.x, rj.y - rj.x, sp, lane, hjx, hjy);
        }
        const float dix = ain.x - ai.x, diy = ain.y - ai.y;
        const float djx = ajn.x - aj.x, djy = ajn.y - aj.y;
        const float dE = -fmaf(dix, hix, -diy * hiy) - fmaf(djx, hjx, -djy * hjy);
        bool accept;
        if (beta_d == 0.0) accept = true;
        else accept = (dE <= 0.f) || (cu < expf(-beta * dE));
        __syncwarp();
        if (accept) {
            sp[i0 * kRepBlock + lane] = ain;
            E += (double)dE;
            nacc++;
        } else {
            sp[j0 * kRepBlock + lane] = aj;
        }
        nprop++;
        if (P.trace != nullptr && U.sample == P.trace_sample && U.rep_begin + lane == P.trace_rep && active) {
            const long long idx = (sw - P.trace_sweep0) * steps + k;
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
        __syncwarp();
    }
    for (int idx = lane; idx < N * kRepBlock; idx += 32) {
        const int site = idx >> 5, l = idx & 31;
        if (l < U.rep_count) P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l] = sp[idx];
    }
    if (active) {
        P.energy[gr] = E;
        P.accepted[gr] += nacc;
        P.proposed[gr] += nprop;
    }
}

size_t resident_smem_bytes_host(int N, int64_t entries) { return resident_smem_bytes(N, entries); }

cudaError_t launch_sweep_resident(const SweepParams& p, int n_units, int variant, int max_N, int64_t max_entries,
                                  cudaStream_t st) {
    if (n_units <= 0) return cudaSuccess;
    const size_t smem = resident_smem_bytes(max_N, max_entries);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    auto kern = variant == 0 ? sweep_resident_kernel<0> : sweep_resident_kernel<1>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<n_units, 32, smem, st>>>(p);
    return cudaGetLastError();
}

}  // namespace pspin
