// internal.h -- engine state shared by the host code and the kernels.
//
// HBM layout of one handle (a batch of S disorder samples):
//
//   spins      float2 [sum_s N_s * R_s]   per sample [site][replica], replica
//                                           fastest, so 32 replicas of one site
//                                           are one 256-byte row
//   per-replica arrays [sum_s R_s]          energy (f64), accepted/proposed
//                                           (i64), beta (f64), RNG key (u64),
//                                           constraint target (f64)
//   site lists int2   [sum_s entries_s]     per sample, per site: groups of
//                                           terms with the same (p, o1), one
//                                           16-byte record {g (f32 bits), o2,
//                                           p<<16|o1, last} per term (or the
//                                           fully connected tiles below), packed
//                                           in TMA chunks of <= 256 entries that
//                                           hold whole groups, start 16-byte
//                                           aligned and have an even length.
//                                           The pair sub-lists of the two-pass
//                                           sweep keep the group format: a
//                                           header {len, p<<16|o1} and len data
//                                           entries {g, o2}
//   chunk starts int64 [n_chunks + 1]       entry offset of every chunk
//   site chunks int32 [sum_s N_s * 33]      first chunk of each of the 32
//                                           balanced parts of a site's list
//                                           (entry 32: one past its last chunk)
//   quartet table Q64 [sum_s nq_s]          active (quartet, channel) with FP64
//                                           g, for the FP64 energy resync
//   g2         f64    [sum_s N_s^2]         dense 2-body couplings (real parts)
//
// Site-list algebra.  For quartet {i,j,k,l} with channel ch the energy term
// is -Re[g a_u1 a_u2 conj(a_c1) conj(a_c2)] (u: unconjugated pair, c:
// conjugated pair; disorder.h:9-16).  For a member site m with partner p
// (the other site of m's pair) and opposite pair {o1,o2}, that term equals
// -Re[a_m * g a_p conj(a_o1) conj(a_o2)] whichever pair m is in, so the
// local field h_m = sum over m's quartets of g a_p conj(a_o1 a_o2) gives
// every energy change of site m alone as -Re[da_m h_m].  2-body terms fold
// in with p = o1 = N, a virtual site whose amplitude is 1.
//
// Fully connected tiles.  When every quartet is active in channel 0, a
// quartet enters site m's field as g a_p conj(a_outer) conj(a_inner) with a
// contiguous range of inner sites shared by every partner p of one outer
// site: if m is among the two smallest sites of the quartet, outer = o1 > m,
// p < o1 and inner in (o1, N); otherwise outer = o2 < m, p > o2 and inner in
// [0, o2).  A tile is a 16-byte header {outer | lo<<16, hi, p0 | p1<<16,
// p2 | p3<<16} and hi-lo rows of 4 couplings (one per partner; padding
// partners are the virtual site with zero couplings), so one gathered
// a_inner feeds 8 FFMA.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pspin {

constexpr int kSplit = 32;        // parts per site list (warps per unit divide it)
constexpr int kGroupMax = 32;     // max data entries after one header
constexpr int kStage = 256;       // max entries per TMA chunk (2 KB)
constexpr int kStages = 3;        // chunks in flight per warp
constexpr int kRepBlock = 32;     // replicas per unit (one per lane)

// Status word bits raised by the sweep kernels.  A CTA (or cluster) whose
// bounded wait ran out stops issuing copies, drains the copies in flight,
// and leaves its replicas' amplitudes, energies and counters as they were
// before the launch.
constexpr int kStatusTimeout = 1;          // a ring wait ran out; the block aborted the launch
constexpr int kStatusDrain = 2;            // the drain of in-flight copies ran out as well
constexpr long long kWaitClocks = 1ll << 31;   // default ring-wait limit (~1 s at 1.9 GHz)
constexpr long long kDrainClocks = 1ll << 31;  // drain limit after an abort

struct SampleDev {
    int N;
    int R;                 // replicas of this sample
    int h2_active;
    int variant;           // 0 sphere (dense), 1 smoothed cube (sparse)
    int fc_tiles;          // 1: site lists are fully connected tiles (see below), 0: group records
    int single_groups;     // group records only, every group of one entry (each record ends its group)
    int64_t spin_off;      // float2 index of site 0, replica 0
    int64_t rep_off;       // index into the per-replica arrays
    int64_t split_off;     // index into site chunks (N*33 entries)
    int64_t q_off;         // index into the Q64 table
    int64_t nq;            // active (quartet, channel) pairs in the Q64 table
    int64_t g2_off;        // index into g2 (N*N doubles)
    int64_t pair_off;      // index into the pair sub-list chunks (N(N-1)*33 entries), -1: not built
    int64_t nb_off;        // index into the neighbour masks (N rows of ceil(N/32) words)
    uint32_t pair_key0, pair_key1;
};

struct Unit {              // one replica block: a CTA, or a cluster of CTAs
    int sample;
    int rep_begin;
    int rep_count;         // <= 32 (32K with K replicas per lane)
    int pad;
};

struct Q64 {               // FP64 quartet for the resync energies
    uint16_t i, j, k, lch; // lch = l | ch << 14
    double g;
};

struct SweepParams {
    const SampleDev* samples;
    const Unit* units;
    float2* spins;
    double* energy;
    long long* accepted;
    long long* proposed;
    const double* beta;
    const uint64_t* key;
    const int2* entries;
    const int64_t* chunk_start;
    const int* site_chunks;
    const int* pair_chunks;           // pair sub-lists (two-pass proposals), or null
    const int* site_chunks_g;         // the site lists in the group format (two-pass proposals;
                                      // tiles unchanged), same per-sample offsets as site_chunks
    const uint32_t* nbmask;           // per sample: row m = sites sharing a quartet (or a g2 term) with m
    const long long* sweep_counter;   // global sweep index at launch start
    int nsweeps;
    int warps;                        // warps per unit (divides 32)
    int cluster;                      // CTAs per unit (sweep_cluster_kernel), 1: sweep_kernel
    // trace
    int trace_sample, trace_rep, trace_cap;
    long long trace_sweep0;
    void* trace;                      // pspin_move_record*
    int* status;                      // error word (kStatus* bits)
    long long wait_clocks;            // ring-wait limit in SM clocks
    int stall_move;                   // tests: move index of the stall wait (-1: none)
};

// shared memory bytes of one sweep CTA: amplitudes, per-warp field
// partials, per-warp chunk rings, ring mbarriers
#ifdef __CUDACC__
__host__ __device__
#endif
inline size_t sweep_smem_bytes(int N, int warps) {
    return (size_t)(N + 1) * kRepBlock * sizeof(float2) + (size_t)warps * kRepBlock * sizeof(float4) +
           (size_t)warps * kStages * kStage * sizeof(int2) + (size_t)warps * kStages * sizeof(uint64_t);
}

// kernels (launchers are host functions in the .cu files)
cudaError_t launch_sweep(const SweepParams& p, int n_units, int variant, int max_N, cudaStream_t st);
cudaError_t launch_sweep_cluster(const SweepParams& p, int n_units, int variant, int max_N, cudaStream_t st,
                                 int* max_clusters);
size_t cluster_smem_bytes_host(int N, int warps, int C);
// the CTA / cluster kernel with K = 2 or 3 replicas per lane (units of up to
// 32K replicas of one sample); cluster 1 launches no cluster
cudaError_t launch_sweep_multi(const SweepParams& p, int n_units, int variant, int max_N, int K, cudaStream_t st,
                               int* max_clusters);
size_t multi_smem_bytes_host(int N, int warps, int C, int K);
// the list-resident kernel; warps > 1 runs batches of consecutive moves that
// commute (no site of one in the other's quartet neighbourhood) on separate
// warps, with the neighbour masks `nbmask`
cudaError_t launch_sweep_resident(const SweepParams& p, int n_units, int variant, int max_N, int64_t max_entries,
                                  cudaStream_t st);
size_t resident_smem_bytes_host(int N, int64_t entries, int warps);

struct EnergyParams {
    const SampleDev* samples;
    const Unit* units;
    float2* spins;
    const Q64* quartets;
    const double* g2;
    double* e2;               // may be null
    double* e4;               // may be null
    double* energy;           // when non-null: running energy <- e2+e4, drift recorded
    double* drift;            // |E_running - E_fp64| before the overwrite (when energy set)
    const double* target;     // constraint target per replica (renormalise when non-null)
    int renorm_only;          // 1: renormalise and return (energies come from elsewhere)
};
cudaError_t launch_energy(const EnergyParams& p, int n_units, int max_N, cudaStream_t st);

struct ExchangeParams {
    int n_samples;
    int NT, nrep;             // per sample
    const SampleDev* samples;
    const double* beta_sched; // [NT]
    const double* energy;
    double* beta;
    int* perm;                // [S][NT*nrep]
    unsigned long long* drand_state; // [S]
    long long* ex_acc;        // [S][NT-1]
    long long* ex_prop;
    long long* sweep_counter; // advanced by nsweeps_done
    int nsweeps_done;
    int do_exchange;
};
cudaError_t launch_exchange(const ExchangeParams& p, cudaStream_t st);

// Observable series at one temperature slot, written after each exchange
// step at row (sweep_counter - sweep0) / pt_freq - 1 (device counter, so a
// captured launch records into the right row).
struct ObserveParams {
    int n_samples, NT, nrep, temp_index, capacity, pt_freq;
    const SampleDev* samples;
    const float2* spins;
    const double* energy;
    const int* perm;
    const long long* sweep_counter;
    long long sweep0;
    double* E_out;            // [capacity][S][nrep]
    double* q_out;            // [capacity][S][nrep*(nrep-1)/2]
};
cudaError_t launch_observe(const ObserveParams& p, cudaStream_t st);

}  // namespace pspin
