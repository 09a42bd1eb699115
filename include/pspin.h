/*
 * pspin.h -- C ABI of the B200 engine for the complex 2+4 p-spin glass.
 *
 * One opaque handle (pspin_state) owns a batch of disorder samples, each
 * with its own N, seed and replicas, resident on one GPU.  A batch of one
 * sample is the reference's MCState / MCStateSparse.  Every entry point
 * returns PSPIN_OK or an error code; pspin_last_error() gives the message.
 * Nothing here calls exit().  Calls on one handle must come from one host
 * thread at a time.  Every call is synchronous with respect to the host
 * unless stated otherwise.
 *
 * Reference interface replaced (giacomotrinca/cuda_pspin), C++ linkage
 * there, extern "C" here:
 *   config.h:9-46, config.cu:6-70   SimConfig, default_config, parse_args
 *   mc.h:33-56                      mc_init, mc_free, mc_sweep, mc_sweep_pt,
 *                                   mc_set_betas, mc_get_results, mc_get_spins,
 *                                   mc_compute_split_energies
 *   mc_sparse.h:42-61               the mc_sparse_* twins
 *   parallel_tempering.cu:316-352   host replica exchange (here on the device)
 *   disorder.h:48-69, disorder.cu   FMC filters and survivor counting
 */
#ifndef PSPIN_H
#define PSPIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------- */
enum {
    PSPIN_OK = 0,
    PSPIN_ERR_ARG = 1,       /* invalid argument (bad N, null pointer, ...)  */
    PSPIN_ERR_CUDA = 2,      /* a CUDA runtime call failed                   */
    PSPIN_ERR_CURAND = 3,    /* a cuRAND call failed                         */
    PSPIN_ERR_ALLOC = 4,     /* device or host allocation failed             */
    PSPIN_ERR_STATE = 5,     /* call not valid in the handle's current state */
    PSPIN_ERR_NUMERIC = 6,   /* running energy left the FP64 resync tolerance */
    PSPIN_ERR_UNSUPPORTED = 7,
    PSPIN_ERR_TIMEOUT = 8    /* a bounded device wait expired: the replica blocks
                                whose wait ran out abandoned that launch and kept
                                their state from before it */
};

enum { PSPIN_DENSE = 0,      /* spherical constraint, dense 3-channel H4 (mc.cu)   */
       PSPIN_SPARSE = 1 };   /* smoothed-cube constraint, N sampled quartets (mc_sparse.cu) */

/* Same field order, types and meaning as the reference's SimConfig
 * (config.h:9-25), so a SimConfig can be passed by address. */
typedef struct pspin_config {
    int save_freq;
    int verbose;
    int N;
    int nrep;            /* replicas in this sample (NT*nrep for PT) */
    double T;
    double J;
    double J0;
    double alpha;
    double alpha0;
    int mc_iterations;
    uint64_t seed;
    int label;
    int dev;
    int fmc_mode;        /* 0 fully connected, 1 comb, 2 uniform */
    double gamma;
} pspin_config;

/* Engine options with no reference counterpart.  Zero-initialised means
 * the defaults (reference-compatible init, resync every 1024 sweeps). */
enum { PSPIN_RESYNC_FP64 = 0, PSPIN_RESYNC_TC = 1 };

typedef struct pspin_options {
    int init_exact;      /* 1: full-sum spin normalisation; 0 (default): the
                            reference's shared-memory tree (spins.cu:27-69),
                            which drops terms for N not a power of two */
    int resync_every;    /* FP64 energy resync + renormalisation period in
                            sweeps (0 -> 1024, <0 -> never) */
    int warps_per_unit;  /* warps sharing one replica block's move; 0 -> auto */
    int trace_sample;    /* record every move of one replica (tests): sample */
    int trace_replica;   /*   ... physical replica; <0 disables tracing */
    int trace_capacity;  /*   ... number of move records kept */
    int quiet;           /* suppress the reference's stdout lines */
    int generic_lists;   /* 1: per-entry site lists for every sample; 0 (default):
                            fully connected dense samples use blocked tiles */
    int graph_steps;     /* pspin_pt_run replays a CUDA graph of this many PT
                            steps (sweeps + exchange); 0 -> 32, <0 -> direct
                            launches.  Results are identical either way. */
    int resync_method;   /* PSPIN_RESYNC_FP64 (default) or PSPIN_RESYNC_TC:
                            periodic energies from the split-BF16 tensor-core
                            contraction (one dense sample per handle) */
    int cluster_size;    /* CTAs (a thread-block cluster) sharing one replica
                            block's lists: 1, 2, 4, 8 or 16 with
                            cluster_size * warps_per_unit <= 32; 0 -> 1;
                            -1: one warp per block with the sample's whole
                            lists resident in shared memory (small lists;
                            plain move only).  Both the plain and the
                            two-pass sweep start with this shape. */
    int wait_limit_clocks; /* the sweep kernels' bounded waits on their copy
                            rings give up after this many SM clocks; 0 ->
                            2^31 (about one second).  A replica block whose
                            wait runs out abandons that launch and keeps its
                            state from before it; the call returns
                            PSPIN_ERR_TIMEOUT. */
    int test_stall_move; /* tests of the time-out path: k > 0 makes every CTA
                            of the ring-fed sweep kernels wait, at move k-1
                            of each launch, on a barrier that nothing
                            completes, so the bounded wait runs out; 0: off */
    int disorder_stream; /* sparse set-up: 0 (default) the reference's couplings
                            bit for bit, from its single cuRAND call of
                            2*C(N,4) normals (2*8*C(N,4) bytes on the device:
                            45 GB at N=512, beyond the device near N=700);
                            1: each selected quartet's coupling from its own
                            counter-based normal (Philox4x32-10 + Box-Muller),
                            the same Gaussian law but not the reference's
                            values, with no C(N,4)-sized memory.  The FMC
                            survivors and the quartet selection are the
                            reference's either way. */
    int replicas_per_lane; /* plain sweep on the CTA / cluster kernels
                            (cluster_size >= 1): 2 or 3 replicas per lane, so
                            one block is 64 or 96 replicas of a sample and
                            every staged coupling serves them all; 1: one
                            replica per lane; 0 (default): 1 until
                            pspin_autotune_lanes picks it.  The chain is the
                            same for every value (same summation order per
                            replica). */
} pspin_options;

typedef struct pspin_info {
    int N;
    int nrep;
    int h2_active;
    int n_quartets;          /* sparse: selected quartets (= N unless fewer survive) */
    int64_t n_pairs_active;  /* g2 non-zeros over i<=j (mc.cu:469-477) */
    int64_t n_quart_active;  /* dense: popcount of the FMC mask; sparse: survivors */
    int64_t site_entries;    /* entries in the per-site sweep lists */
} pspin_info;

/* One recorded move of the traced replica (for per-move dE checks). */
typedef struct pspin_move_record {
    int32_t i0, j0;          /* pair, i0 < j0 */
    float ai_old[2], aj_old[2];
    float ai_new[2], aj_new[2];
    float dE;                /* FP32 dE the kernel accepted or rejected on */
    int32_t accepted;
    float log_q_ratio;       /* log[q(x|x')/q(x'|x)] relative to the plain move (0 for it) */
    float log_u;             /* log of the uniform the decision compared against */
} pspin_move_record;

typedef struct pspin_state pspin_state;

/* ---- configuration (config.h:28-46, config.cu:6-70) --------------- */
void pspin_default_config(pspin_config* cfg);
/* Parses the reference flags into *cfg.  Returns PSPIN_ERR_ARG (and an
 * error message with the usage line) where the reference calls exit(1). */
int  pspin_parse_args(int argc, char** argv, pspin_config* cfg);

/* ---- lifetime (mc_init / mc_sparse_init / mc_free) ------------------- */
int  pspin_create(const pspin_config* cfg, int variant, const pspin_options* opt,
                  pspin_state** out);
/* A batch of independent disorder samples in one handle (each cfg its own
 * N, seed, nrep, FMC).  Sample k's replicas follow sample k-1's in every
 * per-replica array. */
int  pspin_create_batch(const pspin_config* cfgs, int n_samples, int variant,
                        const pspin_options* opt, pspin_state** out);
int  pspin_destroy(pspin_state* s);

/* ---- sweep interface (mc_sweep_pt, mc_set_betas, ...) -------------- */
int  pspin_set_betas(pspin_state* s, const double* betas);      /* [total replicas] */
int  pspin_fill_betas(pspin_state* s, double beta);             /* mc_sweep's 1/T fill */
int  pspin_sweep(pspin_state* s, int nsweeps);                  /* nsweeps x mc_sweep_pt */
int  pspin_get_results(pspin_state* s, double* energies, int64_t* accepted, int64_t* proposed);
int  pspin_reset_counters(pspin_state* s);
int  pspin_get_spins(pspin_state* s, double* spins);             /* [rep][N][re,im] FP64 */
int  pspin_set_spins(pspin_state* s, const double* spins);       /* recomputes energies */
int  pspin_split_energies(pspin_state* s, double* e2, double* e4); /* FP64 from the spins */
int  pspin_resync(pspin_state* s);   /* FP64 energy recompute + constraint renormalisation */
int  pspin_total_replicas(const pspin_state* s);
int  pspin_num_samples(const pspin_state* s);

/* Device pointers into the handle's own per-replica arrays, which the
 * reference's MCState exposes as fields (d_accepted, d_proposed,
 * d_energies, d_betas; mc.h:9-30): int64 accepted and proposed counters,
 * FP64 running energies and betas, [total replicas] each, physical replica
 * order.  Valid until pspin_destroy.  The handle works on its own stream,
 * which does not wait for other streams: work a caller enqueues on these
 * arrays (the reference's drivers cudaMemset the counters,
 * parallel_tempering.cu:396-397) must be complete before the next call on
 * the handle.  Any output pointer may be NULL. */
int  pspin_device_arrays(pspin_state* s, int64_t** accepted, int64_t** proposed, double** energies,
                         double** betas);

/* ---- disorder introspection (MCState fields read by the drivers) ---- */
int  pspin_get_info(pspin_state* s, int sample, pspin_info* info);
int  pspin_get_omega(pspin_state* s, int sample, double* omega); /* [N]; ERR_STATE if FC */
int  pspin_get_couplings(pspin_state* s, int sample, double* g2 /*[N*N*2]*/,
                         double* g4 /*[C(N,4)*2] or NULL*/, uint8_t* mask /*[C(N,4)] or NULL*/);
int  pspin_get_sparse_quartets(pspin_state* s, int sample, int32_t* ijklch /*[n][5]*/, double* g);

/* ---- parallel tempering on the device (parallel_tempering.cu:93-352) */
/* Every sample gets NT temperatures x nrep_per_temp replicas (its nrep must
 * equal NT*nrep_per_temp).  beta_sched[NT], index 0 hottest.  The
 * exchange draws from a drand48 stream seeded like srand48(seed+5000). */
int  pspin_pt_init(pspin_state* s, int NT, int nrep_per_temp, const double* beta_sched,
                   int pt_freq);
/* Runs nsweeps sweeps; after every sweep whose 1-based index is a multiple
 * of pt_freq, proposes the NT-1 adjacent exchanges per replica column. */
int  pspin_pt_run(pspin_state* s, int nsweeps);
/* perm[NT*nrep_per_temp] (logical t*nrep+r -> physical replica) and the
 * cumulative exchange counters [NT-1] of one sample. */
int  pspin_pt_get(pspin_state* s, int sample, int32_t* perm, int64_t* ex_acc, int64_t* ex_prop);
int  pspin_pt_sweeps_done(pspin_state* s, int64_t* sweeps);
/* Host-side replica exchange for drivers that keep the PT loop on the host
 * (the reference's driver pattern, parallel_tempering.cu:316-352) on arrays
 * the caller owns: energy[] and betas[] indexed by rep_off[k] + physical
 * replica, perm[S][NT*nrep] (logical t*nrep+r -> physical), drand_state[S]
 * (48-bit drand48 states, srand48(seed+5000) for the reference's stream),
 * counters ex_acc/ex_prop[S][NT-1]; betas (or NULL) rebuilt from perm. */
int  pspin_exchange_host(int n_samples, int NT, int nrep, const double* beta_sched, const double* energy,
                         const int64_t* rep_off, int32_t* perm, uint64_t* drand_state, int64_t* ex_acc,
                         int64_t* ex_prop, double* betas);
/* Overlap histogram counts of one sample's saved configurations on the GPU
 * (the Parisi P(q) loop of analysis_pt.cpp:1337-1437): configs
 * [nsnap][NT][nrep][N][2] doubles (configs.bin records without the sweep
 * numbers), counts [NT][nbins] of q_ab = Re sum_k a_k conj(b_k) / N over all
 * snapshots and pairs a < b, binned as the reference bins (same rounding, so
 * the same bins). */
int  pspin_overlap_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, double qmin,
                          double qmax, int64_t* counts);
/* Intensity fluctuation overlap histograms of one sample on the GPU (the IFO
 * loop of analysis_pt.cpp:1498-1619 and the experimental IFO of
 * :1679-1806), same configs layout: with I_k = |a_k|^2 and <I_k>_r its mean
 * over the snapshots, IFO bins C_ab = sum_k d_a d_b / sqrt(sum d_a^2 sum
 * d_b^2) of d = I_k - <I_k>_r per snapshot and pair, the experimental IFO
 * the same of d = <I_k>_r - (replica mean of <I_k>_r) once per pair.
 * ifo_counts / exp_counts [NT][nbins], ifo_n / exp_n [NT] the overlaps
 * counted (pairs with a zero norm are skipped, as the reference skips them);
 * either pair of outputs may be NULL.  Binned as the reference bins. */
int  pspin_ifo_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, double cmin,
                      double cmax, int64_t* ifo_counts, int64_t* ifo_n, int64_t* exp_counts, int64_t* exp_n);
/* The deeper analysis of one sample's saved configurations on the GPU
 * (analysis_pt.cpp:1871-2045, run there with --deeper), same configs
 * layout, FP64 in the reference's operation order:
 *   marg [NT][nbins_a2]  counts of I_k = |a_k|^2 in bins of a2_max/nbins_a2
 *                        (kept when inside [0, nbins_a2)), over every
 *                        snapshot, replica and site;
 *   ipr_terms [nsnap][NT][nrep][3]  sum I^2/(sum I)^2, sum I^4/(sum I)^4 and
 *                        1 per configuration ((0, 0, 0) when sum I = 0);
 *   phase, link [NT][nbins]  counts of the phase overlap q_phi (mean of
 *                        cos(theta_a - theta_b) over sites where both
 *                        |.|^2 > 1e-24) and of the link overlap
 *                        q_link = sum_q t_q(a) t_q(b) / M over the M
 *                        quartets [M][5] (i, j, k, l, ch; M = 0: none) per
 *                        snapshot and pair a < b, bins of 2/nbins on [-1, 1];
 *   scatter [NT][nsnap][pairs][2]  (q, q_link) per snapshot and pair. */
int  pspin_deeper_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, int nbins_a2,
                         double a2_max, const int32_t* quartets, int M, int64_t* marg, double* ipr_terms,
                         int64_t* phase, int64_t* link, double* scatter);
/* Multi-overlap values of one sample on the GPU (analysis_pt.cpp:3468-3643):
 * on the snapshots snaps[t][0..nit) of each temperature, out
 * [NT][pairs][nit][3] = (q / sqrt(sum I_a sum I_b), phase overlap over sites
 * with both I > 1e-20, IFO about the mean intensity over those snapshots). */
int  pspin_multi_overlap(int N, int NT, int nrep, int nsnap, const double* configs, const int32_t* snaps,
                         int nit, double* out);
/* The reference's host sampling with the same C++ standard-library engine
 * and distributions, so sampled points and their order are the reference's:
 * idx <- 0..n-1 permuted by std::shuffle with std::mt19937(seed)
 * (analysis_pt.cpp:3504-3507); a reservoir of max_pts points from a stream
 * (std::uniform_int_distribution<int>(0, seen-1), :3609-3619); and per
 * block, when it holds more than max_pts points, a partial Fisher-Yates
 * shuffle with one engine shared by the blocks in order (:2262-2269).
 * Host only; return 0, or 1 on bad arguments. */
int  pspin_std_shuffle(int n, uint32_t seed, int32_t* idx);
int  pspin_reservoir_sample(long long n, int dim, const double* pts, int max_pts, uint32_t seed, double* out,
                            long long* n_out);
int  pspin_fy_downsample(int nblocks, const long long* counts, int dim, const double* pts, int max_pts,
                         uint32_t seed, double* out, long long* out_counts);
/* The reference's energy decorrelation time tau_E of one temperature
 * (analysis_pt.cpp:2703-2752): energy [M][nrep] the saved E/N rows in order;
 * the second half, replica-averaged, and the lag where its autocorrelation
 * first falls below 1/e, linearly interpolated (in save_freq units).  Host
 * only; 0, or 1 on bad arguments. */
int  pspin_tau_e(int M, int nrep, const double* energy, double* tau);
/* NT, replicas per temperature and exchange period set by pspin_pt_init (0s before). */
int  pspin_pt_shape(pspin_state* s, int* NT, int* nrep_per_temp, int* pt_freq);
/* Block-shape autotuner (no reference counterpart): times `sweeps` sweeps
 * for every shape -- the list-resident one-warp kernel (row 0), then
 * clusters of 1, 2, 4, 8, 16 CTAs per replica block x 1, 2, 4, 8 warps per
 * CTA (the resident kernel only for the plain proposal) -- on the handle's
 * own samples, restoring amplitudes, energies, counters and the sweep index
 * after each trial, and keeps the fastest for the current proposal.
 * ms_per_sweep[6][4] (or NULL) receives the timings, -1 where a shape does
 * not fit or does not apply; *chosen_cluster 0 means the resident kernel.
 * The plain sweep keeps its current replicas per lane. */
int  pspin_autotune(pspin_state* s, int sweeps, int* chosen_warps, int* chosen_cluster, float* ms_per_sweep);
/* The same for the plain sweep over 1, 2 and 3 replicas per lane as well:
 * ms_per_sweep[3][6][4] (replicas per lane 1..3, then as above; the resident
 * row applies only to 1).  The chain does not depend on the choice. */
int  pspin_autotune_lanes(pspin_state* s, int sweeps, int* chosen_warps, int* chosen_cluster,
                          int* chosen_replicas_per_lane, float* ms_per_sweep);
/* Observable series at one temperature slot (no reference counterpart; the
 * reference writes E every save_freq sweeps to energy_accept.txt and
 * configurations to configs.bin, parallel_tempering.cu:355-416).  After
 * every exchange step of pspin_pt_run, for every sample: the energies of the
 * nrep replicas at slot temp_index and the overlaps
 * q_ab = Re sum_k a_k^a conj(a_k^b) / N of their nrep(nrep-1)/2 pairs
 * (a < b in slot order).  The first `capacity` steps after the call are
 * kept; capacity 0 switches recording off. */
int  pspin_observe_init(pspin_state* s, int temp_index, int capacity);
/* n_rows: steps recorded (<= capacity); energy [max_rows][S][nrep] and
 * overlap [max_rows][S][nrep(nrep-1)/2] (either may be NULL). */
int  pspin_observe_get(pspin_state* s, int64_t* n_rows, double* energy, double* overlap, int max_rows);

/* ---- all-site local fields (no reference counterpart) ----------------- */
enum { PSPIN_FIELDS_FP64 = 0,      /* FP64 sum over the quartet table */
       PSPIN_FIELDS_TC_BF16X3 = 1  /* tcgen05 contraction, split-BF16 operands, FP32 accumulate */ };
/* Local field h_m of every site of every replica of one dense sample
 * (dE of a one-site change = -Re[da_m h_m]) and the energy computed from
 * the fields.  h [nrep][N][re,im], energy [nrep] (may be NULL).  The
 * tensor-core method builds the symmetric pair-space coupling matrix on its
 * first call for the sample (C(N,2)^2 BF16 x 3 on the device). */
/* |E_running - E_recomputed| per replica (all samples) at the last periodic
 * resync, before the running energy was overwritten. */
int  pspin_resync_drift(pspin_state* s, double* drift);
int  pspin_local_fields(pspin_state* s, int sample, int method, double* h, double* energy);

/* ---- learned pair proposal (no reference counterpart) ----------------- */
/* Proposal used by pspin_sweep / pspin_pt_run (dense variant):
 *   PLAIN         the reference's move (spins.h:17-52), one field pass;
 *   PLAIN_FIELDS  the same move with fields at both ends of every move and,
 *                 after pspin_learn_init, accepted moves recorded for training;
 *   LEARNED       the network's move, accepted with the exact MH ratio
 *                 min(1, e^{-beta dE} [q_L(x|x')/q_P(x|x')]/[q_L(x'|x)/q_P(x'|x)]),
 *                 so the stationary law is the plain chain's. */
enum { PSPIN_PROPOSAL_PLAIN = 0, PSPIN_PROPOSAL_PLAIN_FIELDS = 1, PSPIN_PROPOSAL_LEARNED = 2 };
int  pspin_set_proposal(pspin_state* s, int proposal);
/* Network 8 -> 64 -> 64 -> 26 (tanh), Xavier-initialised from seed; a ring of
 * `capacity` training records (features[8], t', psi_i, psi_j), each accepted
 * PLAIN_FIELDS move being recorded with probability record_prob. */
int  pspin_learn_init(pspin_state* s, uint64_t seed, int capacity, float record_prob);
int  pspin_learn_params(pspin_state* s, float* get /*[6426] or NULL*/, const float* set /*or NULL*/);
/* `steps` Adam steps on minibatches of `batch` records drawn from the ring;
 * mean_loss: mean -log q_L of the last minibatch. */
int  pspin_learn_train(pspin_state* s, int steps, int batch, float lr, double* mean_loss);
int  pspin_learn_records(pspin_state* s, int64_t* n_recorded, float* out /*[max][11] or NULL*/, int max);
/* Loss and gradient of the mean -log q_L over n host records (FP32
 * weights): the check of the backward pass. */
int  pspin_learn_loss_grad(pspin_state* s, const float* records, int n, double* loss, float* grad);

/* ---- checkpoint / resume (no reference counterpart) ------------------ */
/* Everything that continues the chain bit for bit: FP32 amplitudes, running
 * energies, counters, betas, the sweep index that keys the pair and move
 * streams, the resync phase, the PT state (pspin_pt_init's schedule, perm,
 * drand48 states, exchange counters) and the learned network (weights,
 * Adam moments; not the record ring) and the block shapes (which fix the
 * summation order of the fields).  Load into a handle created from the same
 * configurations; anything else is rejected. */
int  pspin_checkpoint_save(pspin_state* s, const char* path);
int  pspin_checkpoint_load(pspin_state* s, const char* path);

/* ---- per-move trace (tests) ------------------------------------------ */
int  pspin_trace_get(pspin_state* s, pspin_move_record* out, int max_records, int* n_records);

/* ---- stand-alone kernels the reference's unit tests exercise --------- */
/* disorder.cu:153-183 on the GPU: first-pass-wins channel mask over C(N,4). */
int  pspin_fmc_mask(int N, const double* omega, double gamma, uint8_t* mask_out,
                    int64_t* n_active);
/* test_quartet_index.cu:56-74 on the GPU: decode -> order -> re-encode for
 * every q < C(N,4); *n_fail counts mismatches. */
int  pspin_quartet_roundtrip(int N, int64_t* n_fail);

/* ---- allocation-free survivor count (no counterpart in the reference) ---
 * For callers that cannot call cudaMalloc (hosts whose own memory pool owns
 * all device memory, plugins handed only device pointers): counts the
 * quartet-channel pairs that pass the FMC filter, like pspin_fmc_mask's
 * n_active, without allocating.  omega[N] and
 * counts[4] (total, channel 0, 1, 2) are device pointers; stream is a
 * cudaStream_t (NULL: the default stream); the call is asynchronous on it.
 * Intermediate per-row counts live in one static device array sized for
 * N <= 1024 (larger N returns PSPIN_ERR_ARG).  The first call on a device
 * (and the first after that device's context was reset) looks up that
 * array's address, and should come before any stream capture.  Calls that
 * overlap on the GPU share the array and race. */
int  pspin_fmc_survivors_static(int N, const double* omega, double gamma, int64_t* counts,
                                void* stream);

/* ---- multi-GPU sharding (no reference counterpart; the reference runs
 * one process per sample, scan_samples_pt:145-169) ---------------------- */
/* Assigns n_samples independent samples (sizes N[k], replicas R[k]) to
 * nshards GPUs by cost N^4 R, largest first to the least-loaded shard.
 * Deterministic: every rank computes the same shard_of[n_samples] alone. */
int  pspin_shard_samples(int n_samples, const int* N, const int* R, int nshards, int* shard_of);

/* ---- the smoothed-cube check (smoothed_cube.cu) ----------------------- */
/* nsamples configurations of N amplitudes on sum |a|^4 = N: one cuRAND
 * Philox call of 2 N nsamples normals from seed, each configuration scaled
 * by (N / sum |a|^4)^(1/4) on the device (smoothed_cube.cu:330-352); out
 * [nsamples][N][2]. */
int  pspin_cube_samples(int N, int nsamples, uint64_t seed, double* out);
/* The free walk of smoothed_cube.cu:74-119 (no Hamiltonian, every move
 * accepted) with the engine's FP32 cube move: start init_spins_cube(seed +
 * 9999) (spins_sparse.cu:63-80), N/2 moves per sweep (the pair (0,1) when
 * N = 2), streams keyed by seed + 12345; traj [max_saved][N][2] holds the
 * start and the state after every save_freq-th sweep, *n_saved their number.
 * The walk is the engine's, so its points are not the reference's; its law
 * (|a_i|^4 / (|a_i|^4 + |a_j|^4) uniform after a move) and the constraint
 * are. */
int  pspin_cube_walk(int N, int sweeps, int save_freq, uint64_t seed, double* traj, int max_saved,
                     int* n_saved);

/* ---- measurement (no reference counterpart) --------------------------- */
/* The CUDA stream (cudaStream_t) all of this handle's work runs on. */
void* pspin_stream(pspin_state* s);
/* When on, every sweep-kernel launch is bracketed by CUDA events on the
 * handle's stream; pspin_get_profile sums their durations since the last
 * call and also reports how many kernels of this library were launched. */
int  pspin_set_profiling(pspin_state* s, int on);
int  pspin_get_profile(pspin_state* s, double* sweep_kernel_ms, int64_t* sweep_launches,
                       int64_t* kernel_launches);
/* Work of one sweep of all samples and replicas (no reference
 * counterpart): algorithmic_flops by the reference method's count per
 * pair-move, F = 20 W4 + 4 W2 + 64 (W4, W2: expected active quartets and
 * off-diagonal pairs touching a random pair), and executed_flops, the FP32
 * operations the local-field kernels actually run on this handle's site
 * lists (about 4 per quartet term and replica) plus the same 64 per move.
 * Either pointer may be NULL. */
int  pspin_sweep_work(pspin_state* s, double* algorithmic_flops, double* executed_flops);
/* FP32 FMA throughput of the current device (TFLOP/s), measured by
 * register-resident FMA loops over all SMs, scalar and paired
 * (fma.rn.f32x2), the faster of the two: the roofline denominator of the
 * FP32 sweep. */
int  pspin_fp32_peak(double* tflops);

/* ---- errors ---------------------------------------------------------- */
const char* pspin_last_error(void);
const char* pspin_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PSPIN_H */
