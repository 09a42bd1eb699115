// rng.cuh -- counter-based random streams used by the engine.
//
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11).  Stateless: a (key, counter) pair maps to
// four 32-bit words, so every replica and every move has its own block and
// a kernel relaunch or a graph replay never needs RNG state in memory.
//
// drand48: the POSIX 48-bit LCG X <- 0x5DEECE66D*X + 0xB (mod 2^48) that
// the reference's host exchange uses (parallel_tempering.cu:304, :334),
// kept on the device so the exchange schedule draws the same stream.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define PSPIN_HD __host__ __device__ __forceinline__
#else
#define PSPIN_HD inline
#endif

namespace pspin {

struct U4 { uint32_t x, y, z, w; };

PSPIN_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
    hi = __umulhi(a, b);
    lo = a * b;
#else
    uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

PSPIN_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Stream tags occupying counter word w, so that the pair schedule, the
// per-replica move stream and set-up draws never share a block.
enum : uint32_t { TAG_PAIR = 0x70616972u, TAG_MOVE = 0x6d6f7665u };

// uniform in [0,1) with 24 random bits (exact in FP32)
PSPIN_HD float u01f(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
// uniform in (0,1] with 24 random bits
PSPIN_HD float u01f_open0(uint32_t x) { return ((float)(x >> 8) + 1.0f) * (1.0f / 16777216.0f); }
// integer in [0, n) by multiply-high (Lemire), bias < n / 2^32
PSPIN_HD uint32_t below(uint32_t x, uint32_t n) {
    return (uint32_t)(((uint64_t)x * n) >> 32);
}

// Pair for step k of sweep s of one sample: i0 uniform in [0,N), j0 uniform
// in the other N-1 sites, returned ordered (the reference's pick,
// mc.cu:129-139, drawn from the sample's shared stream).
PSPIN_HD void pair_pick(uint32_t key0, uint32_t key1, uint64_t sweep, uint32_t k, int N,
                        int& i0, int& j0) {
    U4 c = {k, (uint32_t)sweep, (uint32_t)(sweep >> 32), TAG_PAIR};
    U4 r = philox4x32_10(c, key0, key1);
    int ri = (int)below(r.x, (uint32_t)N);
    int rj = (int)below(r.y, (uint32_t)(N - 1));
    if (rj >= ri) rj++;
    i0 = ri < rj ? ri : rj;
    j0 = ri < rj ? rj : ri;
}

// Four words for one replica's move: proposal (3) and Metropolis (1).
PSPIN_HD U4 move_words(uint32_t key0, uint32_t key1, uint64_t sweep, uint32_t k) {
    U4 c = {k, (uint32_t)sweep, (uint32_t)(sweep >> 32), TAG_MOVE};
    return philox4x32_10(c, key0, key1);
}

// POSIX drand48 on a 48-bit state held in a uint64_t
PSPIN_HD uint64_t srand48_state(long seedval) {
    return (((uint64_t)(uint32_t)seedval) << 16) | 0x330Eu;
}
PSPIN_HD double drand48_next(uint64_t& st) {
    st = (0x5DEECE66DULL * st + 0xBULL) & 0xFFFFFFFFFFFFULL;
    return (double)st * (1.0 / 281474976710656.0);
}

PSPIN_HD uint64_t splitmix64(uint64_t& state) {
    uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace pspin
