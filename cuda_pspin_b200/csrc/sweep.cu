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
#include "internal.h"
#include "rng.cuh"
#include "../../include/pspin.h"

namespace pspin {

template <int VARIANT>
__device__ __forceinline__ void propose(float2 ai, float2 aj, U4 w, float2& ain, float2& ajn) {
    if (VARIANT == 0) {
        // spins.h:17-52: a_i' = a_i e^{-i phi1} sqrt((r1+r2)/r1) cos(alpha),
        //                a_j' = a_j e^{-i phi2} sqrt((r1+r2)/r2) sin(alpha)
        float r1 = fmaf(ai.x, ai.x, ai.y * ai.y);
        float r2 = fmaf(aj.x, aj.x, aj.y * aj.y);
        float sa, ca, s1, c1, s2, c2;
        sincospif(2.0f * u01f(w.x), &sa, &ca);
        sincospif(2.0f * u01f(w.y), &s1, &c1);
        sincospif(2.0f * u01f(w.z), &s2, &c2);
        float s = r1 + r2;
        float f1 = sqrtf(s / r1) * ca;
        float f2 = sqrtf(s / r2) * sa;
        ain = make_float2(fmaf(ai.x, c1, ai.y * s1) * f1, fmaf(ai.y, c1, -ai.x * s1) * f1);
        ajn = make_float2(fmaf(aj.x, c2, aj.y * s2) * f2, fmaf(aj.y, c2, -aj.x * s2) * f2);
    } else {
        // spins_sparse.h:26-56: |a_i'|^2 = sqrt(S4) sqrt(1-u), |a_j'|^2 = sqrt(S4) sqrt(u),
        // absolute phases phi1, phi2
        float u = u01f_open0(w.x);
        float r1 = fmaf(ai.x, ai.x, ai.y * ai.y);
        float r2 = fmaf(aj.x, aj.x, aj.y * aj.y);
        float q = sqrtf(fmaf(r1, r1, r2 * r2));
        float m1 = sqrtf(q * sqrtf(1.0f - u));
        float m2 = sqrtf(q * sqrtf(u));
        float s1, c1, s2, c2;
        sincospif(2.0f * u01f(w.y), &s1, &c1);
        sincospif(2.0f * u01f(w.z), &s2, &c2);
        ain = make_float2(m1 * c1, m1 * s1);
        ajn = make_float2(m2 * c2, m2 * s2);
    }
}

// ---------------------------------------------------------------- TMA ring
// Each warp streams the chunks of its share of the two site lists of every
// move through a ring of kStages shared-memory slots.  Lane 0 issues 1-D
// bulk copies (cp.async.bulk, completion counted on one mbarrier per slot)
// kStages-1 chunks ahead of the chunk being read; the pair schedule is known
// in advance, so the prefetch runs across move boundaries.  Waits are
// bounded: after ~2^31 clocks the kernel sets *status and stops waiting.

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// bounded wait; returns false (and raises the status word) on time-out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) {
            atomicOr(status, 1);
            return false;
        }
    }
    return true;
}

// Position in a warp's chunk stream: move m, list (0: site i0, 1: site j0),
// chunk c of [c, c_end).
struct Cursor {
    int m, which, c, c_end;
};

struct Stream {
    uint32_t key0, key1;
    int N;
    const int* site_chunks;   // this sample's N*(kSplit+1) absolute chunk indices
    long long sweep0;
    int steps, total, part0, part1;

    __device__ __forceinline__ void range(int m, int which, int& c, int& c_end) const {
        int i0, j0;
        const long long sw = sweep0 + m / steps;
        pair_pick(key0, key1, (uint64_t)sw, (uint32_t)(m % steps), N, i0, j0);
        const int* sc = site_chunks + (which ? j0 : i0) * (kSplit + 1);
        c = __ldg(sc + part0);
        c_end = __ldg(sc + part1);
    }
    // move to the next chunk (skipping empty ranges); m == total at the end
    __device__ __forceinline__ void next(Cursor& k) const {
        k.c++;
        while (k.c >= k.c_end) {
            if (++k.which == 2) {
                k.which = 0;
                if (++k.m >= total) return;
            }
            range(k.m, k.which, k.c, k.c_end);
        }
    }
    __device__ __forceinline__ Cursor first() const {
        Cursor k{0, 0, 0, 0};
        if (total <= 0) return k;
        range(0, 0, k.c, k.c_end);
        k.c--;
        next(k);
        return k;
    }
};

// Field contribution of the groups in one staged chunk for this lane's replica.
__device__ __forceinline__ void accumulate_chunk(const int2* __restrict__ R, int n,
                                                 const float2* __restrict__ sp, int lane,
                                                 float& hx, float& hy) {
    int e = 0;
    while (e < n) {
        const int2 h = R[e];
        const int len = h.x;
        const int p = h.y >> 16, o1 = h.y & 0xFFFF;
        const float2 ap = sp[p * kRepBlock + lane];
        const float2 ao = sp[o1 * kRepBlock + lane];
        // a_p * conj(a_o1)
        const float px = fmaf(ap.x, ao.x, ap.y * ao.y);
        const float py = fmaf(ap.y, ao.x, -ap.x * ao.y);
        float yx = 0.f, yy = 0.f;
        const int2* __restrict__ d = R + e + 1;
#pragma unroll 4
        for (int t = 0; t < len; t++) {
            const int2 v = d[t];
            const float g = __int_as_float(v.x);
            const float2 a = sp[v.y * kRepBlock + lane];
            yx = fmaf(g, a.x, yx);       // Y += g conj(a_o2)
            yy = fmaf(-g, a.y, yy);
        }
        hx = fmaf(px, yx, fmaf(-py, yy, hx));
        hy = fmaf(px, yy, fmaf(py, yx, hy));
        e += len + 1;
    }
}

// Field contribution of the fully connected tiles in one staged chunk
// (16-byte records: header, then rows of 4 couplings).  One gathered
// a_inner feeds four partners: 8 FFMA per shared-memory gather.
__device__ __forceinline__ void accumulate_tiles(const int2* __restrict__ R2, int n,
                                                 const float2* __restrict__ sp, int lane,
                                                 float& hx, float& hy) {
    const int4* __restrict__ R = reinterpret_cast<const int4*>(R2);
    const int n16 = n >> 1;
    int e = 0;
    while (e < n16) {
        const int4 hd = R[e];
        const int outer = hd.x & 0xFFFF, lo = hd.x >> 16, hi = hd.y;
        const float2 ao = sp[outer * kRepBlock + lane];
        float y0x = 0.f, y0y = 0.f, y1x = 0.f, y1y = 0.f, y2x = 0.f, y2y = 0.f, y3x = 0.f, y3y = 0.f;
        const float4* __restrict__ C = reinterpret_cast<const float4*>(R + e + 1);
        const float2* __restrict__ A = sp + lo * kRepBlock + lane;
        const int len = hi - lo;
#pragma unroll 2
        for (int t = 0; t < len; t++) {
            const float4 c = C[t];
            const float2 a = A[t * kRepBlock];
            y0x = fmaf(c.x, a.x, y0x); y0y = fmaf(-c.x, a.y, y0y);
            y1x = fmaf(c.y, a.x, y1x); y1y = fmaf(-c.y, a.y, y1y);
            y2x = fmaf(c.z, a.x, y2x); y2y = fmaf(-c.z, a.y, y2y);
            y3x = fmaf(c.w, a.x, y3x); y3y = fmaf(-c.w, a.y, y3y);
        }
        // h += sum_k a_pk conj(a_outer) Y_k
        const int pk[4] = {hd.z & 0xFFFF, hd.z >> 16, hd.w & 0xFFFF, hd.w >> 16};
        const float yx[4] = {y0x, y1x, y2x, y3x}, yy[4] = {y0y, y1y, y2y, y3y};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float2 ap = sp[pk[k] * kRepBlock + lane];
            const float px = fmaf(ap.x, ao.x, ap.y * ao.y);
            const float py = fmaf(ap.y, ao.x, -ap.x * ao.y);
            hx = fmaf(px, yx[k], fmaf(-py, yy[k], hx));
            hy = fmaf(px, yy[k], fmaf(py, yx[k], hy));
        }
        e += 1 + len;
    }
}

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

    for (int idx = threadIdx.x; idx < N * kRepBlock; idx += blockDim.x) {
        const int site = idx >> 5, l = idx & 31;
        float2 v = make_float2(1.f, 0.f);
        if (l < U.rep_count) v = P.spins[S.spin_off + (int64_t)site * R + U.rep_begin + l];
        sp[idx] = v;
    }
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

    Stream st;
    st.key0 = S.pair_key0;
    st.key1 = S.pair_key1;
    st.N = N;
    st.site_chunks = P.site_chunks + S.split_off;
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

    __syncthreads();
    if (warp == 0 && total > 0) prepare(0);
    __syncthreads();

    for (int m = 0; m < total; m++) {
        const long long sw = sweep0 + m / steps;
        const int k = m % steps;
        float h[4] = {0.f, 0.f, 0.f, 0.f};
        for (int which = 0; which < 2; which++) {
            int c, c_end;
            st.range(m, which, c, c_end);
            for (; c < c_end; c++) {
                const uint32_t slot = consumed % kStages;
                if (ok) ok = mbar_wait(bars + slot, (consumed / kStages) & 1u, P.status);
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
        __syncthreads();

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
                }
            }
            if (m + 1 < total) prepare(m + 1);
        }
        __syncthreads();
    }
    // copies still in flight after a time-out: wait for them (bounded)
    if (!ok && lane == 0)
        for (uint32_t k = consumed; k < issued; k++) mbar_wait(bars + k % kStages, (k / kStages) & 1u, P.status);

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
