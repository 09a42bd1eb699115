// sweep_common.cuh -- device pieces shared by the sweep kernels: proposals,
// the per-warp TMA rings that stream site-list chunks into shared memory,
// and the field accumulation over one staged chunk.
#pragma once
#include "internal.h"
#include "rng.cuh"

namespace pspin {

// The state-independent part of a move's proposal, from its four random
// words: t[0], t[1] = sin, cos of the rotation angle (sphere) or
// sqrt(1-u), sqrt(u) of the transfer (cube); t[2..5] = sin, cos of the two
// phases; t[6] = the Metropolis uniform.
template <int VARIANT>
__device__ __forceinline__ void move_trig(U4 w, float* t) {
    if (VARIANT == 0) {
        sincospif(2.0f * u01f(w.x), &t[0], &t[1]);
    } else {
        const float u = u01f_open0(w.x);
        t[0] = sqrtf(1.0f - u);
        t[1] = sqrtf(u);
    }
    sincospif(2.0f * u01f(w.y), &t[2], &t[3]);
    sincospif(2.0f * u01f(w.z), &t[4], &t[5]);
    t[6] = u01f(w.w);
}

// The state-dependent part: the proposed amplitudes from the current ones.
template <int VARIANT>
__device__ __forceinline__ void propose_with(float2 ai, float2 aj, const float* t, float2& ain, float2& ajn) {
    const float s1 = t[2], c1 = t[3], s2 = t[4], c2 = t[5];
    if (VARIANT == 0) {
        // spins.h:17-52: a_i' = a_i e^{-i phi1} sqrt((r1+r2)/r1) cos(alpha),
        //                a_j' = a_j e^{-i phi2} sqrt((r1+r2)/r2) sin(alpha)
        const float sa = t[0], ca = t[1];
        float r1 = fmaf(ai.x, ai.x, ai.y * ai.y);
        float r2 = fmaf(aj.x, aj.x, aj.y * aj.y);
        float s = r1 + r2;
        float f1 = sqrtf(s / r1) * ca;
        float f2 = sqrtf(s / r2) * sa;
        ain = make_float2(fmaf(ai.x, c1, ai.y * s1) * f1, fmaf(ai.y, c1, -ai.x * s1) * f1);
        ajn = make_float2(fmaf(aj.x, c2, aj.y * s2) * f2, fmaf(aj.y, c2, -aj.x * s2) * f2);
    } else {
        // spins_sparse.h:26-56: |a_i'|^2 = sqrt(S4) sqrt(1-u), |a_j'|^2 = sqrt(S4) sqrt(u),
        // absolute phases phi1, phi2
        float r1 = fmaf(ai.x, ai.x, ai.y * ai.y);
        float r2 = fmaf(aj.x, aj.x, aj.y * aj.y);
        float q = sqrtf(fmaf(r1, r1, r2 * r2));
        float m1 = sqrtf(q * t[0]);
        float m2 = sqrtf(q * t[1]);
        ain = make_float2(m1 * c1, m1 * s1);
        ajn = make_float2(m2 * c2, m2 * s2);
    }
}

template <int VARIANT>
__device__ __forceinline__ void propose(float2 ai, float2 aj, U4 w, float2& ain, float2& ajn) {
    float t[7];
    move_trig<VARIANT>(w, t);
    propose_with<VARIANT>(ai, aj, t, ain, ajn);
}

// Static shared memory of the ring-fed cluster kernels (ring tags, the
// stall-test barrier), kept free in their dynamic-size accounting.
constexpr size_t kStaticSmem = 256;

// ---------------------------------------------------------------- block state
// Prologue copies into shared memory with kInFlight independent loads per
// thread before their stores, so a CTA's state arrives in a few memory
// latencies rather than one per loop trip.
constexpr int kInFlight = 8;

// A replica block's amplitudes: columns [0, kb) of rows [0, N) of the
// sample's [site][R] array `src` (already offset to the block's first
// replica) into sp[site * kb + col]; columns >= rep_count are 1+0i.
__device__ __forceinline__ void load_block_amplitudes(float2* sp, const float2* src, int64_t R, int N, int kb,
                                                      int rep_count) {
    const int total = N * kb;
    const int step = (int)blockDim.x;
    for (int i0 = threadIdx.x; i0 < total; i0 += kInFlight * step) {
        float2 v[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; u++) {
            const int idx = i0 + u * step;
            const int site = idx / kb, col = idx - site * kb;
            v[u] = make_float2(1.f, 0.f);
            if (idx < total && col < rep_count) v[u] = src[site * R + col];
        }
#pragma unroll
        for (int u = 0; u < kInFlight; u++) {
            const int idx = i0 + u * step;
            if (idx < total) sp[idx] = v[u];
        }
    }
}

// n contiguous elements
template <class T>
__device__ __forceinline__ void load_block_range(T* dst, const T* src, int64_t n) {
    const int64_t step = blockDim.x;
    for (int64_t i0 = threadIdx.x; i0 < n; i0 += kInFlight * step) {
        T v[kInFlight];
#pragma unroll
        for (int u = 0; u < kInFlight; u++) {
            const int64_t idx = i0 + u * step;
            if (idx < n) v[u] = src[idx];
        }
#pragma unroll
        for (int u = 0; u < kInFlight; u++) {
            const int64_t idx = i0 + u * step;
            if (idx < n) dst[idx] = v[u];
        }
    }
}

// ---------------------------------------------------------------- TMA ring
// Each warp streams the chunks of its share of the two site lists of every
// move through a ring of kStages shared-memory slots.  Lane 0 issues 1-D
// bulk copies (cp.async.bulk, completion counted on one mbarrier per slot)
// kStages-1 chunks ahead of the chunk being read; the pair schedule is known
// in advance, so the prefetch runs across move boundaries.  Waits are
// bounded (SweepParams::wait_clocks): a wait that runs out raises the status
// word, and the CTA (every CTA of a cluster) aborts the launch at the next
// move barrier without writing anything back.

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

// Bounded wait; returns false and raises `flag` in the status word when
// `limit` SM clocks pass before the phase completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, long long limit,
                                          int flag = kStatusTimeout) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            atomicOr(status, flag);
            return false;
        }
    }
    return true;
}

// A ring wait made warp-uniform: the warp goes on only if every lane saw
// the copy land.
__device__ __forceinline__ bool ring_wait(uint64_t* bar, uint32_t parity, int* status, long long limit) {
    return __all_sync(0xffffffffu, mbar_wait(bar, parity, status, limit));
}

// After an abort: lane 0 waits (bounded) for the copies this warp issued and
// never consumed, so that no bulk copy is still writing into shared memory
// when the CTA exits.  Completed phases pass at once (their parity is the
// previous phase's), so a copy whose wait gave up is waited for again here.
__device__ __forceinline__ void drain_ring(uint64_t* bars, int stages, uint32_t consumed, uint32_t issued,
                                           int* status) {
    if ((threadIdx.x & 31) == 0)
        for (uint32_t q = consumed; q < issued; q++)
            if (!mbar_wait(bars + q % stages, (q / stages) & 1u, status, kDrainClocks, kStatusDrain)) break;
    __syncwarp();
}

// Test hook: the bounded wait of every warp at move P.stall_move on an
// mbarrier that nothing arrives on, so the wait runs out and the kernel
// takes its abort path.
__device__ __forceinline__ bool stall_wait(uint64_t* bar, int* status, long long limit) {
    return ring_wait(bar, 0u, status, limit);
}

// Position in a warp's chunk stream: move m, list (0: site i0, 1: site j0),
// chunk c of [c, c_end).
struct Cursor {
    int m, which, c, c_end;
};

// kLists: lists visited per move -- sites i0, j0 (2); then, for the two-pass
// sweep, the pair's two sub-lists (4).  kCache: keep the last pair pick of the
// consumer and of the cursor (fewer Philox evaluations, two more live
// registers; measured faster for sweep_kernel and the two-pass sweep, slower
// for the cluster sweep)
template <int kLists, bool kCache = true>
struct Stream {
    uint32_t key0, key1;
    int N;
    const int* site_chunks;   // this sample's N*(kSplit+1) absolute chunk indices
    const int* pair_chunks;   // this sample's N(N-1)*(kSplit+1) pair sub-list chunk indices
    long long sweep0;
    int steps, total, part0, part1;
    // the last pair pick of the consumer (slot 0) and of the prefetch cursor
    // (slot 1): each list lookup of a move reuses it instead of another Philox
    int cm[2] = {-1, -1}, ci[2] = {0, 0}, cj[2] = {0, 0};

    __device__ __forceinline__ void range(int m, int which, int& c, int& c_end, int slot = 0) {
        int i0, j0;
        if (kCache) {
            if (m != cm[slot]) {
                const long long sw = sweep0 + m / steps;
                pair_pick(key0, key1, (uint64_t)sw, (uint32_t)(m % steps), N, ci[slot], cj[slot]);
                cm[slot] = m;
            }
            i0 = ci[slot];
            j0 = cj[slot];
        } else {
            const long long sw = sweep0 + m / steps;
            pair_pick(key0, key1, (uint64_t)sw, (uint32_t)(m % steps), N, i0, j0);
        }
        const int* sc = (kLists == 2 || which < 2) ? site_chunks + ((which & 1) ? j0 : i0) * (kSplit + 1)
                                                   : pair_chunks + (2 * (j0 * (j0 - 1) / 2 + i0) + (which & 1)) * (kSplit + 1);
        c = __ldg(sc + part0);
        c_end = __ldg(sc + part1);
    }
    // move to the next chunk (skipping empty ranges); m == total at the end
    __device__ __forceinline__ void next(Cursor& k) {
        k.c++;
        while (k.c >= k.c_end) {
            if (++k.which == kLists) {
                k.which = 0;
                if (++k.m >= total) return;
            }
            range(k.m, k.which, k.c, k.c_end, 1);
        }
    }
    __device__ __forceinline__ Cursor first() {
        Cursor k{0, 0, 0, 0};
        if (total <= 0) return k;
        range(0, 0, k.c, k.c_end, 1);
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

// The same groups stored as 16-byte records {g, o2, p<<16|o1, last}, one
// per data entry: a record's position does not depend on an earlier header.
// Records are taken kUnroll at a time with their shared-memory loads (the
// records, then each record's a_o2, a_p, a_o1, the last two used only where
// the record ends a group) issued before the arithmetic, so a batch costs
// about two load latencies: for chains that wait on latency (a few warps
// per SM).  Kernels that fill the SMs use accumulate_records_k's one record
// at a time, which loads a_p, a_o1 once per group.  The arithmetic is
// accumulate_chunk's, operation for operation: Y accumulates the group's
// entries in order from zero and h takes a_p conj(a_o1) Y at the group's
// last record.  kSingle: every record ends its group (groups of one entry,
// the rule for sparse samples), so the test is compiled out.
template <bool kSingle>
__device__ __forceinline__ void record_step(const int4 q, const float2 a, const float2 ap, const float2 ao,
                                            float& yx, float& yy, float& hx, float& hy) {
    const float g = __int_as_float(q.x);
    yx = fmaf(g, a.x, yx);               // Y += g conj(a_o2)
    yy = fmaf(-g, a.y, yy);
    if (kSingle || q.w) {
        const float px = fmaf(ap.x, ao.x, ap.y * ao.y);
        const float py = fmaf(ap.y, ao.x, -ap.x * ao.y);
        hx = fmaf(px, yx, fmaf(-py, yy, hx));
        hy = fmaf(px, yy, fmaf(py, yx, hy));
        yx = 0.f;
        yy = 0.f;
    }
}

template <int kUnroll = 4, bool kSingle = false>
__device__ __forceinline__ void accumulate_records(const int2* __restrict__ R2, int n,
                                                   const float2* __restrict__ sp, int lane,
                                                   float& hx, float& hy) {
    const int4* __restrict__ R = reinterpret_cast<const int4*>(R2);
    const int nr = n >> 1;
    float yx = 0.f, yy = 0.f;
    int r = 0;
    for (; r + kUnroll <= nr; r += kUnroll) {
        int4 q[kUnroll];
        float2 a[kUnroll], ap[kUnroll], ao[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) q[u] = R[r + u];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            a[u] = sp[q[u].y * kRepBlock + lane];
            ap[u] = sp[(q[u].z >> 16) * kRepBlock + lane];
            ao[u] = sp[(q[u].z & 0xFFFF) * kRepBlock + lane];
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) record_step<kSingle>(q[u], a[u], ap[u], ao[u], yx, yy, hx, hy);
    }
    for (; r < nr; r++) {
        const int4 q = R[r];
        record_step<kSingle>(q, sp[q.y * kRepBlock + lane], sp[(q.z >> 16) * kRepBlock + lane],
                             sp[(q.z & 0xFFFF) * kRepBlock + lane], yx, yy, hx, hy);
    }
}

// Field contribution of the fully connected tiles in one staged chunk
// (16-byte records: header, then rows of 4 couplings).  One gathered
// a_inner feeds four partners: 8 FFMA per shared-memory gather.  The rows
// are unrolled by kUnroll (more gathers in flight per warp; the summation
// order is the same for every kUnroll).
template <int kUnroll = 8>
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
#pragma unroll kUnroll
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

// ---------------------------------------------------------------- K replicas per lane
// The same accumulations for a block of 32K replicas stored [site][K][32]
// (replica k*32 + lane of the block at sp[(site*K + k)*32 + lane]): each
// staged coupling is read once and used for the lane's K replicas.  The
// summation order per replica is that of accumulate_tiles /
// accumulate_records.
template <int K, int kUnroll>
__device__ __forceinline__ void accumulate_tiles_k(const int2* __restrict__ R2, int n,
                                                   const float2* __restrict__ sp, int lane,
                                                   float (&hx)[K], float (&hy)[K]) {
    const int4* __restrict__ R = reinterpret_cast<const int4*>(R2);
    const int n16 = n >> 1;
    int e = 0;
    while (e < n16) {
        const int4 hd = R[e];
        const int outer = hd.x & 0xFFFF, lo = hd.x >> 16, hi = hd.y;
        float y[K][8];
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
            for (int q = 0; q < 8; q++) y[k][q] = 0.f;
        const float4* __restrict__ C = reinterpret_cast<const float4*>(R + e + 1);
        const float2* __restrict__ A = sp + (size_t)lo * K * kRepBlock + lane;
        const int len = hi - lo;
#pragma unroll kUnroll
        for (int t = 0; t < len; t++) {
            const float4 c = C[t];
#pragma unroll
            for (int k = 0; k < K; k++) {
                const float2 a = A[(t * K + k) * kRepBlock];
                y[k][0] = fmaf(c.x, a.x, y[k][0]); y[k][1] = fmaf(-c.x, a.y, y[k][1]);
                y[k][2] = fmaf(c.y, a.x, y[k][2]); y[k][3] = fmaf(-c.y, a.y, y[k][3]);
                y[k][4] = fmaf(c.z, a.x, y[k][4]); y[k][5] = fmaf(-c.z, a.y, y[k][5]);
                y[k][6] = fmaf(c.w, a.x, y[k][6]); y[k][7] = fmaf(-c.w, a.y, y[k][7]);
            }
        }
        const int pk[4] = {hd.z & 0xFFFF, hd.z >> 16, hd.w & 0xFFFF, hd.w >> 16};
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float2 ao = sp[(outer * K + k) * kRepBlock + lane];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float2 ap = sp[(pk[q] * K + k) * kRepBlock + lane];
                const float px = fmaf(ap.x, ao.x, ap.y * ao.y);
                const float py = fmaf(ap.y, ao.x, -ap.x * ao.y);
                hx[k] = fmaf(px, y[k][2 * q], fmaf(-py, y[k][2 * q + 1], hx[k]));
                hy[k] = fmaf(px, y[k][2 * q + 1], fmaf(py, y[k][2 * q], hy[k]));
            }
        }
        e += 1 + len;
    }
}

// One record at a time (accumulate_records_k for one replica per lane).
__device__ __forceinline__ void accumulate_records_1(const int2* __restrict__ R2, int n,
                                                     const float2* __restrict__ sp, int lane, float& hx, float& hy);

template <int K>
__device__ __forceinline__ void accumulate_records_k(const int2* __restrict__ R2, int n,
                                                     const float2* __restrict__ sp, int lane,
                                                     float (&hx)[K], float (&hy)[K]) {
    const int4* __restrict__ R = reinterpret_cast<const int4*>(R2);
    const int nr = n >> 1;
    float yx[K], yy[K];
#pragma unroll
    for (int k = 0; k < K; k++) yx[k] = yy[k] = 0.f;
#pragma unroll 4
    for (int r = 0; r < nr; r++) {
        const int4 q = R[r];
        const float g = __int_as_float(q.x);
#pragma unroll
        for (int k = 0; k < K; k++) {
            const float2 a = sp[(q.y * K + k) * kRepBlock + lane];
            yx[k] = fmaf(g, a.x, yx[k]);
            yy[k] = fmaf(-g, a.y, yy[k]);
        }
        if (q.w) {
            const int p = q.z >> 16, o1 = q.z & 0xFFFF;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const float2 ap = sp[(p * K + k) * kRepBlock + lane];
                const float2 ao = sp[(o1 * K + k) * kRepBlock + lane];
                const float px = fmaf(ap.x, ao.x, ap.y * ao.y);
                const float py = fmaf(ap.y, ao.x, -ap.x * ao.y);
                hx[k] = fmaf(px, yx[k], fmaf(-py, yy[k], hx[k]));
                hy[k] = fmaf(px, yy[k], fmaf(py, yx[k], hy[k]));
                yx[k] = 0.f;
                yy[k] = 0.f;
            }
        }
    }
}

__device__ __forceinline__ void accumulate_records_1(const int2* __restrict__ R2, int n,
                                                     const float2* __restrict__ sp, int lane, float& hx, float& hy) {
    float hx1[1] = {hx}, hy1[1] = {hy};
    accumulate_records_k<1>(R2, n, sp, lane, hx1, hy1);
    hx = hx1[0];
    hy = hy1[0];
}

// The field partials of the C CTAs x W warps of a block, summed in the fixed
// order the cluster kernels use -- each CTA's warps in order, then the CTAs
// in rank order -- from slots buf[(q*W + w) * stride], with the loads of
// four slots in flight before their additions (the same additions in the
// same order as one load per addition).
__device__ __forceinline__ void add4v(float4& a, const float4 b) {
    a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w;
}
__device__ __forceinline__ float4 sum_partials(const float4* buf, int C, int W, int stride) {
    float4 hs = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int q = 0; q < C; q++) {
        float4 part = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int w0 = 0; w0 < W; w0 += 4) {
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (w0 + u < W) v[u] = buf[(size_t)(q * W + w0 + u) * stride];
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (w0 + u < W) {
                    if (w0 + u == 0) part = v[u];
                    else add4v(part, v[u]);
                }
        }
        if (q == 0) hs = part;
        else add4v(hs, part);
    }
    return hs;
}

// ---------------------------------------------------------------- clusters
// Partial fields of the CTAs of a thread-block cluster meet in every CTA's
// exchange buffer (distributed shared memory).
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// store v into the same shared-memory location of CTA `rank` of the cluster
__device__ __forceinline__ void st_cluster_f4(const void* local, uint32_t rank, float4 v) {
    const uint32_t la = (uint32_t)__cvta_generic_to_shared(local);
    uint32_t ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"(rank));
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(ra), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ void st_cluster_u32(const void* local, uint32_t rank, uint32_t v) {
    const uint32_t la = (uint32_t)__cvta_generic_to_shared(local);
    uint32_t ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(la), "r"(rank));
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(ra), "r"(v) : "memory");
}

}  // namespace pspin
