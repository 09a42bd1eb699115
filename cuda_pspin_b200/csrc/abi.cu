// abi.cu -- the extern "C" boundary (include/pspin.h) and host orchestration.
//
// mc_init / mc_sparse_init (mc.cu:411-562, mc_sparse.cu:390-604) become
// pspin_create_batch: the same cuRAND host-API calls with the same seeds
// produce the same FP64 disorder and initial amplitudes; FMC masks and
// survivor counts run on the device; the sweep layout is built on the host.
#include <cuda_runtime.h>
#include <curand.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <chrono>
#include <unordered_map>
#include <vector>

#include "../../include/pspin.h"
#include "internal.h"
#include "layout.h"
#include "rng.cuh"

#include <cuda_bf16.h>

namespace pspin {
cudaError_t tc_gemm(int M, int NC, int K3, const __nv_bfloat16* A, const __nv_bfloat16* B, float* F, void* workspace,
                    size_t ws_bytes, cudaStream_t st, size_t* ws_needed);
cudaError_t launch_split_ws(const float* ws, __nv_bfloat16* out, int M, int Kp, cudaStream_t st);
cudaError_t launch_pair_split(const float2* spins, int N, int R, int npairs, int Kp, __nv_bfloat16* X,
                              cudaStream_t st);
cudaError_t launch_site_fields(const float2* spins, int N, int R, const float* F, int NC, const double* g2,
                               int h2_active, float2* h, double* e2, double* e4, cudaStream_t st);
cudaError_t launch_fp64_fields(const float2* spins, int N, int R, const Q64* Q, int64_t nq, const double* g2,
                               int h2_active, double2* h, cudaStream_t st);
struct LearnParams {
    int mode;
    const __nv_bfloat16* w;
    float* records;
    unsigned long long* rec_count;
    int rec_cap;
    float rec_prob;
};
cudaError_t launch_learned_sweep(const SweepParams& p, const LearnParams& l, int n_units, int max_N, cudaStream_t st,
                                 int* max_clusters);
size_t learned_smem_bytes_host(int N, int warps, int C);
cudaError_t launch_mlp_fwd_bwd(const float* w, const float* records, const int* index, int n, float* save,
                               float* loss, cudaStream_t st);
cudaError_t launch_mlp_grad(const float* save, int n, float* grad, cudaStream_t st);
cudaError_t launch_adam(float* w, float* m, float* v, const float* g, __nv_bfloat16* wbf, float lr, int t,
                        cudaStream_t st);
cudaError_t launch_to_bf16(const float* w, __nv_bfloat16* wbf, cudaStream_t st);
cudaError_t launch_sample_index(int* idx, int n, unsigned long long filled, uint64_t key, uint32_t step,
                                cudaStream_t st);
constexpr int kMlpParamsHost = 6426, kRecordFloatsHost = 11, kSaveFloatsHost = 8 + 4 * 64 + 26;
cudaError_t dev_fmc_mask(uint8_t* mask, const double* omega, int N, double gamma, cudaStream_t st);
cudaError_t launch_cube_normalize_many(double* all, int N, int nsamples, cudaStream_t st);
cudaError_t dev_g2_build(const double* normals, int N, const double* omega, double gamma, double* g2,
                         unsigned long long* count, cudaStream_t st);
cudaError_t dev_g2_scale(double* g2, long long n, double sigma, double mean, int shift, cudaStream_t st);
cudaError_t dev_normalize_replicas(const double* nrm, int N, int R, int cube, int exact, float2* spins,
                                   double* target, cudaStream_t st);
cudaError_t launch_cube_walk(float2* a, int N, int sweeps, int save_freq, uint64_t move_key, uint64_t pair_key,
                             double* traj, int max_saved, int* n_saved, cudaStream_t st);
cudaError_t dev_survivor_counts(unsigned long long* counts, const double* omega, int N, double gamma, cudaStream_t st);
cudaError_t dev_popcount(const uint8_t* mask, int64_t n, unsigned long long* out, cudaStream_t st);
cudaError_t dev_g4_real(const double* normals, double* g4, int64_t n, double sigma, double mean, cudaStream_t st);
cudaError_t dev_gather_real(const double* normals, const int64_t* qs, int n, double* out, cudaStream_t st);
cudaError_t dev_roundtrip(int N, int64_t nq, unsigned long long* fails, cudaStream_t st);
}  // namespace pspin

using namespace pspin;

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

namespace pspin {
int report_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
}  // namespace pspin

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(PSPIN_ERR_CUDA, "CUDA error at %s:%d: %s", __FILE__, __LINE__,             \
                        cudaGetErrorString(e_));                                                     \
    } while (0)

#define CKR(call)                                                                                    \
    do {                                                                                             \
        curandStatus_t e_ = (call);                                                                  \
        if (e_ != CURAND_STATUS_SUCCESS)                                                             \
            return fail(PSPIN_ERR_CURAND, "cuRAND error at %s:%d: %d", __FILE__, __LINE__, (int)e_); \
    } while (0)

#define TRY(call)                      \
    do {                               \
        int rc_ = (call);              \
        if (rc_ != PSPIN_OK) return rc_; \
    } while (0)

template <class T>
static int dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return PSPIN_OK;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(PSPIN_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    }
    return PSPIN_OK;
}

// ------------------------------------------------------------------ state
struct SampleHost {
    pspin_config cfg;
    int N = 0, R = 0;
    std::vector<double> omega;
    std::vector<double> g2re;        // N*N (real parts; imag is 0)
    int64_t n_pairs_active = 0, n_quart_active = 0;
    int h2_active = 0;
    std::vector<int32_t> sq;         // sparse: [n][5]
    std::vector<double> sqg;
    int64_t site_entries = 0;
    double exec_flops_lists = 0.0;   // FP32 ops per replica to accumulate all N site lists once
    int64_t g4_off = -1;             // dense: into d_g4re / d_mask
    int fc_tiles = 0;                // site lists are fully connected tiles (else group records)
    int single_groups = 0;           // group records, every group of one entry
    int64_t nq_dense = 0;
};

struct pspin_state {
    int variant = 0;
    int S = 0;
    pspin_options opt{};
    std::vector<SampleHost> hs;
    std::vector<SampleDev> sd;
    std::vector<Unit> units;
    int R_tot = 0, max_N = 0, warps = 8, cluster = 1;   // cluster 0: list-resident one-warp kernel
    int64_t max_site_entries = 0;
    int warps2 = 8, cluster2 = 1;       // block shape of the two-pass (learned / fields) sweep
    int rpl = 1;                        // replicas per lane of the plain CTA / cluster sweep
    std::vector<Unit> units_k[2];       // blocks of 64 and 96 replicas (rpl 2, 3)
    int64_t spin_total = 0;
    cudaStream_t st = nullptr;
    int device = 0;

    SampleDev* d_samples = nullptr;
    Unit* d_units = nullptr;
    Unit* d_units_k[2] = {nullptr, nullptr};
    float2* d_spins = nullptr;
    double *d_E = nullptr, *d_beta = nullptr, *d_target = nullptr, *d_drift = nullptr, *d_e2 = nullptr,
           *d_e4 = nullptr;
    long long *d_acc = nullptr, *d_prop = nullptr;
    uint64_t* d_key = nullptr;
    int2* d_entries = nullptr;
    int64_t* d_chunk_start = nullptr;
    int* d_site_chunks = nullptr;
    int* d_pair_chunks = nullptr;       // pair sub-lists, built on the first two-pass proposal
    int* d_site_chunks_g = nullptr;     // site lists in the group format, built with the pair sub-lists
    uint32_t* d_nbmask = nullptr;       // per sample: neighbour masks (rows of ceil(N/32) words)
    int64_t ent_total = 0, chunk_total = 0;
    Q64* d_q64 = nullptr;
    double* d_g2 = nullptr;
    double* d_g4re = nullptr;
    uint8_t* d_mask = nullptr;
    long long* d_sweep_counter = nullptr;
    int* d_status = nullptr;

    // parallel tempering
    int pt_NT = 0, pt_nrep = 0, pt_freq = 0;
    double* d_beta_sched = nullptr;
    int* d_perm = nullptr;
    unsigned long long* d_drand = nullptr;
    long long *d_ex_acc = nullptr, *d_ex_prop = nullptr;

    // tensor-core all-site fields (one sample at a time)
    int tc_sample = -1, tc_M = 0, tc_Kp = 0, tc_NC = 0;
    __nv_bfloat16* d_tc_w = nullptr;     // [M][3Kp]
    __nv_bfloat16* d_tc_x = nullptr;     // [NC][3Kp]
    float* d_tc_f = nullptr;             // [M][NC]
    void* d_tc_ws = nullptr;
    size_t tc_ws_bytes = 0;
    float2* d_tc_h = nullptr;
    double2* d_f64_h = nullptr;
    double* d_tc_e = nullptr;            // [2][R]

    // learned proposal
    int proposal = PSPIN_PROPOSAL_PLAIN;
    float *d_w32 = nullptr, *d_adam_m = nullptr, *d_adam_v = nullptr, *d_grad = nullptr;
    __nv_bfloat16* d_wbf = nullptr;
    float* d_records = nullptr;
    unsigned long long* d_rec_count = nullptr;
    int rec_cap = 0;
    float rec_prob = 0.f;
    float *d_save = nullptr, *d_loss = nullptr;
    int* d_idx = nullptr;
    int save_cap = 0;
    int adam_t = 0;
    uint64_t learn_seed = 0;

    // observable series at one temperature slot
    double *d_obs_E = nullptr, *d_obs_q = nullptr;
    int obs_t = -1, obs_cap = 0;
    long long obs_sweep0 = 0;

    // trace
    pspin_move_record* d_trace = nullptr;
    long long trace_sweep0 = 0;

    long long sweeps_done = 0;
    long long since_resync = 0;

    // CUDA graph of graph_G PT steps (pspin_pt_run), rebuilt when a captured
    // pointer or kernel choice changes
    cudaGraphExec_t graph_exec = nullptr;
    int graph_G = 0;
    long long graph_launches = 0;

    // measurement
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    size_t ev_used = 0;
    long long sweep_launches = 0, kernel_launches = 0;
};

static void free_state(pspin_state* s) {
    if (!s) return;
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    void* ptrs[] = {s->d_samples, s->d_units, s->d_spins, s->d_E, s->d_beta, s->d_target, s->d_drift,
                    s->d_e2, s->d_e4, s->d_acc, s->d_prop, s->d_key, s->d_entries, s->d_chunk_start, s->d_site_chunks,
                    s->d_q64, s->d_g2, s->d_g4re, s->d_mask, s->d_sweep_counter, s->d_status,
                    s->d_beta_sched, s->d_perm, s->d_drand, s->d_ex_acc, s->d_ex_prop, s->d_trace,
                    s->d_tc_w, s->d_tc_x, s->d_tc_f, s->d_tc_ws, s->d_tc_h, s->d_f64_h, s->d_tc_e,
                    s->d_w32, s->d_adam_m, s->d_adam_v, s->d_grad, s->d_wbf, s->d_records, s->d_rec_count,
                    s->d_save, s->d_loss, s->d_idx, s->d_obs_E, s->d_obs_q, s->d_pair_chunks, s->d_site_chunks_g, s->d_nbmask,
                    s->d_units_k[0], s->d_units_k[1]};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& e : s->ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
}

// ------------------------------------------------------------------ config
extern "C" void pspin_default_config(pspin_config* c) {
    // config.h:28-46
    std::memset(c, 0, sizeof(*c));
    c->N = 64;
    c->nrep = 1;
    c->T = 1.0;
    c->J = 2.0;
    c->J0 = 0.0;
    c->alpha = 0.5;
    c->alpha0 = 0.5;
    c->mc_iterations = 10000;
    c->seed = 42;
    c->save_freq = 100;
    c->verbose = 0;
    c->label = -1;
    c->dev = -1;
    c->fmc_mode = 0;
    c->gamma = 0.0;
}

extern "C" int pspin_parse_args(int argc, char** argv, pspin_config* cfg) {
    // config.cu:6-70, with exit(1) replaced by PSPIN_ERR_ARG
    if (!cfg) return fail(PSPIN_ERR_ARG, "null config");
    pspin_default_config(cfg);
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        bool has = i + 1 < argc;
        if (!strcmp(a, "-N") && has) cfg->N = atoi(argv[++i]);
        else if (!strcmp(a, "-nrep") && has) cfg->nrep = atoi(argv[++i]);
        else if (!strcmp(a, "-T") && has) cfg->T = atof(argv[++i]);
        else if (!strcmp(a, "-J") && has) cfg->J = atof(argv[++i]);
        else if (!strcmp(a, "-J0") && has) cfg->J0 = atof(argv[++i]);
        else if (!strcmp(a, "-alpha") && has) cfg->alpha = atof(argv[++i]);
        else if (!strcmp(a, "-alpha0") && has) cfg->alpha0 = atof(argv[++i]);
        else if (!strcmp(a, "-iter") && has) cfg->mc_iterations = atoi(argv[++i]);
        else if (!strcmp(a, "-seed") && has) cfg->seed = strtoull(argv[++i], nullptr, 10);
        else if (!strcmp(a, "-save_freq") && has) cfg->save_freq = atoi(argv[++i]);
        else if (!strcmp(a, "-label") && has) cfg->label = atoi(argv[++i]);
        else if (!strcmp(a, "-dev") && has) cfg->dev = atoi(argv[++i]);
        else if (!strcmp(a, "-fmc") && has) cfg->fmc_mode = atoi(argv[++i]);
        else if (!strcmp(a, "-gamma") && has) cfg->gamma = atof(argv[++i]);
        else if (!strcmp(a, "-verbose")) {
            if (i + 1 < argc && argv[i + 1][0] >= '0' && argv[i + 1][0] <= '9') cfg->verbose = atoi(argv[++i]);
            else cfg->verbose = 1;
        } else {
            return fail(PSPIN_ERR_ARG,
                        "Unknown argument: %s\nUsage: %s [-N n] [-nrep n] [-T temp] [-J coupling] [-J0 mean] "
                        "[-alpha a] [-alpha0 a0] [-iter n] [-seed s] [-save_freq k] [-label l] [-dev d] "
                        "[-fmc 0|1|2] [-gamma g] [-verbose [0|1|2]]",
                        a, argc > 0 ? argv[0] : "pspin");
        }
    }
    if (cfg->N < 4) return fail(PSPIN_ERR_ARG, "Error: N must be >= 4 for 4-body interactions.");
    if (cfg->fmc_mode > 0 && cfg->gamma <= 0.0) {
        if (cfg->fmc_mode == 1) cfg->gamma = 0.0;
        else if (cfg->fmc_mode == 2) cfg->gamma = 1.0 / (2.0 * (cfg->N - 1));
    }
    return PSPIN_OK;
}

// ------------------------------------------------------------------ set-up helpers
static inline int64_t C4(int64_t n) { return n * (n - 1) * (n - 2) * (n - 3) / 24; }
static inline int64_t C3(int64_t n) { return n * (n - 1) * (n - 2) / 6; }
static inline int64_t C2(int64_t n) { return n * (n - 1) / 2; }

struct Curand {
    curandGenerator_t g = nullptr;
    ~Curand() {
        if (g) curandDestroyGenerator(g);
    }
};

// curandGenerateNormalDouble(PHILOX4_32_10, seed) into device memory; a fresh
// generator per call, as in disorder.cu:61-68 and spins.cu:75-82
static int curand_normals(uint64_t seed, size_t count, double* d_out, cudaStream_t st) {
    Curand c;
    CKR(curandCreateGenerator(&c.g, CURAND_RNG_PSEUDO_PHILOX4_32_10));
    CKR(curandSetStream(c.g, st));
    CKR(curandSetPseudoRandomGeneratorSeed(c.g, seed));
    CKR(curandGenerateNormalDouble(c.g, d_out, count, 0.0, 1.0));
    return PSPIN_OK;
}

static void omega_of(const pspin_config& c, std::vector<double>& w) {
    // mc.cu:449-460
    w.resize(c.N);
    if (c.fmc_mode == 1) {
        for (int i = 0; i < c.N; i++) w[i] = (double)i;
    } else {
        uint64_t st = c.seed + 3000;
        for (int i = 0; i < c.N; i++) {
            uint64_t z = splitmix64(st);
            w[i] = (double)(z >> 11) / (double)(1ULL << 53);
        }
        std::sort(w.begin(), w.end());
    }
}

// g2 generation, FMC, survivor count, rescale, mean shift
// (mc.cu:443-444, 465-478, 491-498; disorder.cu:57-91, 130-143)
// g2 on the device (disorder.cu:45-80, 130-143, 191-197; mc.cu:436-502):
// cuRAND normals (seed + 1000), real parts, symmetric copy, FMC filter and
// survivor count (i <= j, the diagonal always survives), then sigma =
// J2 sqrt(N / n) and the mean shift on the non-zero entries; the host keeps
// a copy for the layouts.
static int setup_g2(SampleHost& h, cudaStream_t st) {
    const pspin_config& c = h.cfg;
    const int N = c.N;
    const double J2 = (1.0 - c.alpha) * c.J, J20 = (1.0 - c.alpha0) * c.J0;
    h.g2re.assign((size_t)N * N, 0.0);
    if (c.fmc_mode > 0) omega_of(c, h.omega);
    else h.omega.clear();
    if (c.fmc_mode == 1) {                 // comb: H2 fully killed
        h.n_pairs_active = 0;
        h.h2_active = 0;
        return PSPIN_OK;
    }
    double *d = nullptr, *d_g2 = nullptr, *d_w = nullptr;
    unsigned long long* d_cnt = nullptr;
    int rc = dalloc(&d, 2 * (size_t)N * N);
    if (rc == PSPIN_OK) rc = dalloc(&d_g2, (size_t)N * N);
    if (rc == PSPIN_OK) rc = dalloc(&d_w, (size_t)N);
    if (rc == PSPIN_OK) rc = dalloc(&d_cnt, 1);
    if (rc == PSPIN_OK) rc = curand_normals(c.seed + 1000, 2 * (size_t)N * N, d, st);
    unsigned long long cnt = 0;
    if (rc == PSPIN_OK) {
        cudaError_t e = cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st);
        if (e == cudaSuccess && c.fmc_mode == 2)
            e = cudaMemcpyAsync(d_w, h.omega.data(), N * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = dev_g2_build(d, N, c.fmc_mode == 2 ? d_w : nullptr, c.gamma, d_g2, d_cnt, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) {
            h.n_pairs_active = c.fmc_mode == 2 ? (int64_t)cnt : (int64_t)N * (N + 1) / 2;
            const double sigma = h.n_pairs_active > 0 ? J2 * std::sqrt((double)N / (double)h.n_pairs_active) : 1.0;
            const double mean = (J20 != 0.0 && h.n_pairs_active > 0) ? J20 * (double)N / (double)h.n_pairs_active : 0.0;
            e = dev_g2_scale(d_g2, (long long)N * N, sigma, mean, mean != 0.0 ? 1 : 0, st);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h.g2re.data(), d_g2, (size_t)N * N * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "g2 set-up: %s", cudaGetErrorString(e));
    }
    cudaFree(d);
    cudaFree(d_g2);
    cudaFree(d_w);
    cudaFree(d_cnt);
    h.h2_active = h.n_pairs_active > 0 ? 1 : 0;
    return rc;
}

// spins.cu:27-69 (sphere) / spins_sparse.cu:28-61 (cube), on the host in
// FP64.  Returns the constraint value of the normalised amplitudes.
static double normalize_host(double* sp, int N, int cube, int exact) {
    if (!cube) {
        double norm = 0.0;
        if (exact || N > 1024) {
            for (int i = 0; i < N; i++) norm += sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1];
        } else {
            std::vector<double> s(N);
            for (int t = 0; t < N; t++) s[t] = sp[2 * t] * sp[2 * t] + sp[2 * t + 1] * sp[2 * t + 1];
            for (int w = N / 2; w > 0; w >>= 1)
                for (int t = 0; t < w; t++) s[t] += s[t + w];
            norm = s[0];
        }
        const double scale = std::sqrt((double)N / norm);
        for (int i = 0; i < 2 * N; i++) sp[i] *= scale;
        double r = 0.0;
        for (int i = 0; i < N; i++) r += sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1];
        return r;
    }
    int bd = (N < 1024) ? ((N + 31) / 32 * 32) : 1024;
    if (bd < 32) bd = 32;
    double sum = 0.0;
    if (exact) {
        for (int i = 0; i < N; i++) {
            const double r2 = sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1];
            sum += r2 * r2;
        }
    } else {
        std::vector<double> s(bd, 0.0);
        for (int t = 0; t < bd && t < N; t++) {
            const double r2 = sp[2 * t] * sp[2 * t] + sp[2 * t + 1] * sp[2 * t + 1];
            s[t] = r2 * r2;
        }
        for (int w = bd / 2; w > 0; w >>= 1)
            for (int t = 0; t < w; t++) s[t] += s[t + w];
        sum = s[0];
    }
    const double scale = std::pow((double)N / sum, 0.25);
    const int lim = exact ? N : std::min(N, bd);
    for (int i = 0; i < 2 * lim; i++) sp[i] *= scale;
    double r = 0.0;
    for (int i = 0; i < N; i++) {
        const double r2 = sp[2 * i] * sp[2 * i] + sp[2 * i + 1] * sp[2 * i + 1];
        r += r2 * r2;
    }
    return r;
}

// The idx-th survivor (q*3+ch, in ascending order) given survivor counts of
// the (l,k) blocks and their prefix sums.
struct SurvivorIndex {
    int N = 0;
    int fmc = 0;
    double gamma = 0.0;
    const double* w = nullptr;
    std::vector<int> bl, bk;          // non-empty blocks in q order
    std::vector<int64_t> pre;         // prefix (size blocks+1)
    int64_t total = 0;

    int64_t at(int64_t idx) const {
        if (fmc == 0) return idx * 3;          // every quartet, channel 0
        size_t b = std::upper_bound(pre.begin(), pre.end(), idx) - pre.begin() - 1;
        const int l = bl[b], k = bk[b];
        int64_t left = idx - pre[b];
        const int64_t base = C4(l) + C3(k);
        int64_t p = 0;
        for (int j = 1; j < k; j++)
            for (int i = 0; i < j; i++, p++) {
                const double wi = w[i], wj = w[j], wk = w[k], wl = w[l];
                uint8_t m = 0;
                if (std::fabs(wi + wj - wk - wl) <= gamma) m = 1;
                else if (std::fabs(wi + wl - wj - wk) <= gamma) m = 2;
                else if (std::fabs(wi + wk - wj - wl) <= gamma) m = 4;
                for (int ch = 0; ch < 3; ch++)
                    if (m & (1 << ch)) {
                        if (left == 0) return (base + p) * 3 + ch;
                        left--;
                    }
            }
        return -1;
    }
};

static void decode_q(int64_t q, int& i, int& j, int& k, int& l) {
    // mc_sparse.cu:320-335
    int ll = 3;
    while (C4(ll) <= q) ll++;
    ll--;
    int64_t rem = q - C4(ll);
    int kk = 2;
    while (C3(kk) <= rem) kk++;
    kk--;
    rem -= C3(kk);
    int jj = 1;
    while (C2(jj) <= rem) jj++;
    jj--;
    rem -= C2(jj);
    i = (int)rem; j = jj; k = kk; l = ll;
}

// mc_sparse.cu:477-537 without the dense temporaries: survivors are counted
// per (l,k) block on the device and the partial Fisher-Yates shuffle runs on
// a virtual array whose entries are located by rank.
// Standard normal of quartet q for the streamed sparse set-up: Philox4x32-10
// (rng.cuh) keyed by splitmix64 of the coupling seed, counter (q, TAG_G4),
// two 53-bit uniforms u1 in (0, 1], u2 in [0, 1) and the Box-Muller transform
// z = sqrt(-2 ln u1) cos(2 pi u2) (Box & Muller, Ann. Math. Statist. 29, 610,
// 1958).  Host arithmetic; independent of every other quartet's draw.
static double quartet_normal(uint64_t seed, int64_t q) {
    uint64_t st = seed;
    const uint64_t key = splitmix64(st);
    const U4 w = philox4x32_10(U4{(uint32_t)q, (uint32_t)((uint64_t)q >> 32), 0u, 0x67346e72u},
                               (uint32_t)key, (uint32_t)(key >> 32));
    const uint64_t m1 = ((uint64_t)w.x << 32) | w.y, m2 = ((uint64_t)w.z << 32) | w.w;
    const double u1 = ((double)(m1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = (double)(m2 >> 11) * (1.0 / 9007199254740992.0);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

static int setup_sparse_quartets(pspin_state* s, SampleHost& h, std::vector<QuartetRec>& qs) {
    const pspin_config& c = h.cfg;
    const int N = c.N;
    const double J4 = c.alpha * c.J, J40 = c.alpha0 * c.J0;
    const int64_t nq = C4(N);
    SurvivorIndex si;
    si.N = N;
    si.fmc = c.fmc_mode;
    si.gamma = c.gamma;
    si.w = h.omega.data();
    if (c.fmc_mode == 0) {
        si.total = nq;
    } else {
        double* d_w = nullptr;
        unsigned long long* d_cnt = nullptr;
        TRY(dalloc(&d_w, N));
        int rc = dalloc(&d_cnt, (size_t)N * N);
        std::vector<unsigned long long> cnt((size_t)N * N);
        if (rc == PSPIN_OK) {
            cudaError_t e = cudaMemcpyAsync(d_w, h.omega.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->st);
            if (e == cudaSuccess) e = dev_survivor_counts(d_cnt, d_w, N, c.gamma, s->st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(cnt.data(), d_cnt, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
            if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "survivor count: %s", cudaGetErrorString(e));
        }
        cudaFree(d_w);
        cudaFree(d_cnt);
        if (rc != PSPIN_OK) return rc;
        si.pre.push_back(0);
        for (int l = 3; l < N; l++)
            for (int k = 2; k < l; k++) {
                const unsigned long long v = cnt[(size_t)l * N + k];
                if (!v) continue;
                si.bl.push_back(l);
                si.bk.push_back(k);
                si.pre.push_back(si.pre.back() + (int64_t)v);
            }
        si.total = si.pre.back();
    }
    h.n_quart_active = si.total;
    int ns = N;
    if (si.total < ns) {
        if (!s->opt.quiet)
            fprintf(stderr, "WARNING: only %lld non-zero quartets after FMC, requested %d. Using all.\n",
                    (long long)si.total, ns);
        ns = (int)si.total;
    }
    // partial Fisher-Yates (mc_sparse.cu:340-349) on the virtual survivor array
    std::unordered_map<int64_t, int64_t> moved;
    auto get = [&](int64_t i) {
        auto it = moved.find(i);
        return it != moved.end() ? it->second : si.at(i);
    };
    uint64_t rng = c.seed + 4000;
    const int64_t count = si.total;
    for (int i = 0; i < ns && i < (int)count; i++) {
        const uint64_t r = splitmix64(rng);
        const int64_t j = i + (int64_t)(r % (uint64_t)(count - i));
        const int64_t vi = get(i), vj = get(j);
        moved[i] = vj;
        moved[j] = vi;
    }
    std::vector<int64_t> sel(ns), selq(ns);
    for (int t = 0; t < ns; t++) {
        sel[t] = get(t);
        selq[t] = sel[t] / 3;
    }
    // coupling values: the same single cuRAND call as the reference's dense
    // temporary (mc_sparse.cu:424, disorder.cu:93-106), gathered at the
    // selected quartets; or, with disorder_stream, one counter-based normal
    // per selected quartet (no C(N,4)-sized memory, not the reference's values)
    std::vector<double> raw(ns);
    if (ns > 0 && s->opt.disorder_stream) {
        for (int t = 0; t < ns; t++) raw[t] = quartet_normal(c.seed + 2000 + 12345, selq[t]);
    } else if (ns > 0) {
        double* d_nrm = nullptr;
        int64_t* d_q = nullptr;
        double* d_out = nullptr;
        int rc = dalloc(&d_nrm, 2 * (size_t)nq);
        if (rc != PSPIN_OK)
            return fail(PSPIN_ERR_ALLOC,
                        "sparse set-up needs the cuRAND stream of 2*C(N,4) = %lld doubles on the device (%s); "
                        "options.disorder_stream = 1 draws the selected couplings without it (same law, "
                        "not the reference's values)",
                        (long long)(2 * nq), g_err.c_str());
        rc = dalloc(&d_q, ns);
        if (rc == PSPIN_OK) rc = dalloc(&d_out, ns);
        if (rc == PSPIN_OK) rc = curand_normals(c.seed + 2000 + 12345, 2 * (size_t)nq, d_nrm, s->st);
        if (rc == PSPIN_OK) {
            cudaError_t e = cudaMemcpyAsync(d_q, selq.data(), ns * sizeof(int64_t), cudaMemcpyHostToDevice, s->st);
            if (e == cudaSuccess) e = dev_gather_real(d_nrm, d_q, ns, d_out, s->st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(raw.data(), d_out, ns * sizeof(double), cudaMemcpyDeviceToHost, s->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
            if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "sparse gather: %s", cudaGetErrorString(e));
        }
        cudaFree(d_nrm);
        cudaFree(d_q);
        cudaFree(d_out);
        if (rc != PSPIN_OK) return rc;
    }
    const double sigma = J4 * std::sqrt((double)N / (double)(ns > 0 ? ns : 1));
    const double mean4 = (J40 != 0.0) ? J40 * (double)N / (double)ns : 0.0;
    h.sq.resize((size_t)ns * 5);
    h.sqg.resize(ns);
    qs.clear();
    for (int t = 0; t < ns; t++) {
        const int ch = (int)(sel[t] % 3);
        int i, j, k, l;
        decode_q(selq[t], i, j, k, l);
        const double g = raw[t] * sigma + mean4;
        int32_t* e = &h.sq[(size_t)t * 5];
        e[0] = i; e[1] = j; e[2] = k; e[3] = l; e[4] = ch;
        h.sqg[t] = g;
        qs.push_back(QuartetRec{i, j, k, l, ch, g});
    }
    return PSPIN_OK;
}

// dense g4: generation, FMC mask, popcount, rescale, shift, all on the
// device (mc.cu:445-446, 480-483, 492, 499-502)
static int setup_dense_g4(pspin_state* s, SampleHost& h, std::vector<double>& g4re, std::vector<uint8_t>& mask) {
    const pspin_config& c = h.cfg;
    const int N = c.N;
    const int64_t nq = C4(N);
    const double J4 = c.alpha * c.J, J40 = c.alpha0 * c.J0;
    double* d_nrm = nullptr;
    TRY(dalloc(&d_nrm, 2 * (size_t)nq));
    int rc = curand_normals(c.seed + 2000 + 12345, 2 * (size_t)nq, d_nrm, s->st);
    double* g4 = s->d_g4re + h.g4_off;
    uint8_t* m = s->d_mask + h.g4_off;
    unsigned long long* d_cnt = nullptr;
    double* d_w = nullptr;
    if (rc == PSPIN_OK) rc = dalloc(&d_cnt, 1);
    if (rc == PSPIN_OK && c.fmc_mode > 0) rc = dalloc(&d_w, N);
    if (rc == PSPIN_OK) {
        cudaError_t e = cudaSuccess;
        unsigned long long a = 0;
        if (c.fmc_mode > 0) {
            e = cudaMemcpyAsync(d_w, h.omega.data(), N * sizeof(double), cudaMemcpyHostToDevice, s->st);
            if (e == cudaSuccess) e = dev_fmc_mask(m, d_w, N, c.gamma, s->st);
            if (e == cudaSuccess) e = dev_popcount(m, nq, d_cnt, s->st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&a, d_cnt, sizeof(a), cudaMemcpyDeviceToHost, s->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
        } else {
            e = cudaMemsetAsync(m, 1, (size_t)nq, s->st);
            a = (unsigned long long)nq;
        }
        h.n_quart_active = (int64_t)a;
        if (e == cudaSuccess) {
            const double sigma = (a > 0) ? J4 * std::sqrt((double)N / (double)a) : 1.0;
            const double mean = (J40 != 0.0 && a > 0) ? J40 * (double)N / (double)a : 0.0;
            e = dev_g4_real(d_nrm, g4, nq, sigma, mean, s->st);
        }
        if (e == cudaSuccess) {
            g4re.resize(nq);
            mask.resize(nq);
            e = cudaMemcpyAsync(g4re.data(), g4, nq * sizeof(double), cudaMemcpyDeviceToHost, s->st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(mask.data(), m, nq, cudaMemcpyDeviceToHost, s->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
        }
        if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "dense g4 set-up: %s", cudaGetErrorString(e));
    }
    cudaFree(d_nrm);
    cudaFree(d_cnt);
    cudaFree(d_w);
    return rc;
}

static int choose_warps(const pspin_state* s) {
    if (s->opt.warps_per_unit > 0) {
        int w = s->opt.warps_per_unit;
        if (w > 8 || (32 % w) != 0) return -1;
        return w;
    }
    double per_site = 0.0;
    for (const SampleHost& h : s->hs) per_site = std::max(per_site, (double)h.site_entries / h.N);
    if (per_site > 16000) return 8;
    if (per_site > 4000) return 4;
    if (per_site > 1000) return 2;
    return 1;
}

static int run_energy(pspin_state* s, double* e2, double* e4, bool overwrite, bool renorm) {
    EnergyParams p{};
    p.samples = s->d_samples;
    p.units = s->d_units;
    p.spins = s->d_spins;
    p.quartets = s->d_q64;
    p.g2 = s->d_g2;
    p.e2 = e2;
    p.e4 = e4;
    p.energy = overwrite ? s->d_E : nullptr;
    p.drift = overwrite ? s->d_drift : nullptr;
    p.target = renorm ? s->d_target : nullptr;
    CK(launch_energy(p, (int)s->units.size(), s->max_N, s->st));
    s->kernel_launches++;
    return PSPIN_OK;
}

extern "C" int pspin_create_batch(const pspin_config* cfgs, int n, int variant, const pspin_options* opt,
                                  pspin_state** out) {
    if (!cfgs || n <= 0 || !out) return fail(PSPIN_ERR_ARG, "pspin_create_batch: bad arguments");
    if (variant != PSPIN_DENSE && variant != PSPIN_SPARSE) return fail(PSPIN_ERR_ARG, "unknown variant %d", variant);
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        const pspin_config& c = cfgs[k];
        if (c.N < 4) return fail(PSPIN_ERR_ARG, "Error: N must be >= 4 for 4-body interactions.");
        if (c.N > 1000) return fail(PSPIN_ERR_ARG, "N=%d above the engine limit 1000", c.N);
        if (c.nrep < 1) return fail(PSPIN_ERR_ARG, "nrep must be >= 1");
        if (c.fmc_mode < 0 || c.fmc_mode > 2) return fail(PSPIN_ERR_ARG, "fmc must be 0, 1 or 2");
        if (variant == PSPIN_DENSE && C4(c.N) > (int64_t)400000000)
            return fail(PSPIN_ERR_ARG, "dense variant: C(N,4) too large for N=%d", c.N);
    }
    pspin_state* s = new pspin_state();
    if (opt) s->opt = *opt;
    else {
        std::memset(&s->opt, 0, sizeof(s->opt));
        s->opt.trace_replica = -1;
    }
    if (s->opt.resync_every == 0) s->opt.resync_every = 1024;
    if (s->opt.resync_method != PSPIN_RESYNC_FP64 && s->opt.resync_method != PSPIN_RESYNC_TC) {
        const int m = s->opt.resync_method;
        delete s;
        return fail(PSPIN_ERR_ARG, "unknown resync method %d", m);
    }
    if (s->opt.resync_method == PSPIN_RESYNC_TC && (variant != PSPIN_DENSE || n != 1)) {
        delete s;
        return fail(PSPIN_ERR_UNSUPPORTED, "the tensor-core resync takes one dense sample per handle");
    }
    s->variant = variant;
    s->S = n;
    s->hs.resize(n);
    auto bail = [&](int rc) {
        free_state(s);
        return rc;
    };
    {
        int dev = cfgs[0].dev;
        if (dev >= 0) {
            cudaError_t e = cudaSetDevice(dev);
            if (e != cudaSuccess) return bail(fail(PSPIN_ERR_CUDA, "cudaSetDevice(%d): %s", dev, cudaGetErrorString(e)));
        }
        cudaGetDevice(&s->device);
        cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bail(fail(PSPIN_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    }

    // ---- per-sample host descriptors and pools
    int64_t g4_pool = 0;
    for (int k = 0; k < n; k++) {
        SampleHost& h = s->hs[k];
        h.cfg = cfgs[k];
        h.N = cfgs[k].N;
        h.R = cfgs[k].nrep;
        if (variant == PSPIN_DENSE) {
            h.g4_off = g4_pool;
            h.nq_dense = C4(h.N);
            g4_pool += h.nq_dense;
        }
        s->R_tot += h.R;
        s->max_N = std::max(s->max_N, h.N);
        s->spin_total += (int64_t)h.N * h.R;
    }
    int rc = PSPIN_OK;
    if (variant == PSPIN_DENSE) {
        rc = dalloc(&s->d_g4re, (size_t)g4_pool);
        if (rc == PSPIN_OK) rc = dalloc(&s->d_mask, (size_t)g4_pool);
        if (rc != PSPIN_OK) return bail(rc);
    }

    // ---- disorder, spins, layouts
    std::vector<SiteLists> lists(n);
    std::vector<std::vector<Q64>> q64(n);
    std::vector<std::vector<uint64_t>> keys(n);
    const bool timing = std::getenv("PSPIN_SETUP_TIMING") != nullptr;
    auto clk = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
        return std::chrono::duration<double>(b - a).count();
    };
    const auto t_p1 = clk();
    // phase 1 (device, in sample order): cuRAND streams, FMC masks, survivor
    // counts, coupling rescale; host copies of what the layout needs
    std::vector<std::vector<QuartetRec>> qsv(n);
    std::vector<std::vector<double>> g4h(n);
    std::vector<std::vector<uint8_t>> maskh(n);
    // each sample's replica normals stay on the device until the normalisation
    // kernel writes them, scaled, into the amplitude array
    struct DevNormals {
        std::vector<double*> p;
        ~DevNormals() {
            for (double* x : p) cudaFree(x);
        }
    } nrm_dev;
    nrm_dev.p.assign(n, nullptr);
    for (int k = 0; k < n; k++) {
        SampleHost& h = s->hs[k];
        const int N = h.N, R = h.R;
        rc = setup_g2(h, s->st);
        if (rc != PSPIN_OK) return bail(rc);
        if (variant == PSPIN_DENSE) {
            rc = setup_dense_g4(s, h, g4h[k], maskh[k]);
            if (rc != PSPIN_OK) return bail(rc);
        } else {
            rc = setup_sparse_quartets(s, h, qsv[k]);
            if (rc != PSPIN_OK) return bail(rc);
        }
        // replica seeds (mc.cu:419-423) double as the Philox move keys (mc.cu:521)
        keys[k].resize(R);
        uint64_t master = h.cfg.seed;
        for (int r = 0; r < R; r++) keys[k][r] = splitmix64(master);
        // initial amplitudes: cuRAND normals per replica (spins.cu:75-82)
        {
            double*& d = nrm_dev.p[k];
            rc = dalloc(&d, 2 * (size_t)N * R);
            if (rc != PSPIN_OK) return bail(rc);
            // one generator, re-seeded with its offset reset for every
            // replica: the stream of a fresh generator with that seed
            Curand c;
            curandStatus_t cs = curandCreateGenerator(&c.g, CURAND_RNG_PSEUDO_PHILOX4_32_10);
            if (cs == CURAND_STATUS_SUCCESS) cs = curandSetStream(c.g, s->st);
            for (int r = 0; r < R && cs == CURAND_STATUS_SUCCESS; r++) {
                cs = curandSetPseudoRandomGeneratorSeed(c.g, keys[k][r]);
                if (cs == CURAND_STATUS_SUCCESS) cs = curandSetGeneratorOffset(c.g, 0);
                if (cs == CURAND_STATUS_SUCCESS)
                    cs = curandGenerateNormalDouble(c.g, d + 2 * (size_t)N * r, 2 * (size_t)N, 0.0, 1.0);
            }
            if (cs != CURAND_STATUS_SUCCESS) rc = fail(PSPIN_ERR_CURAND, "spin init cuRAND error %d", (int)cs);
            if (rc != PSPIN_OK) return bail(rc);
        }
    }
    const auto t_p2 = clk();
    // phase 2 (host, samples in parallel): quartet lists, per-site sweep
    // lists, FP64 quartet tables
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < n; k++) {
        SampleHost& h = s->hs[k];
        const int N = h.N;
        bool fc = false;
        if (variant == PSPIN_DENSE) {
            dense_quartets(N, g4h[k].data(), maskh[k].data(), qsv[k]);
            // fully connected tiles when every quartet is active in channel 0
            fc = !s->opt.generic_lists && h.cfg.fmc_mode == 0 && (int64_t)qsv[k].size() == C4(N);
            for (const QuartetRec& r : qsv[k])
                if (!fc || r.ch != 0) { fc = false; break; }
            if (fc) build_site_tiles_fc(N, h.g2re.data(), h.h2_active, g4h[k].data(), lists[k]);
            std::vector<double>().swap(g4h[k]);
            std::vector<uint8_t>().swap(maskh[k]);
        }
        h.fc_tiles = fc ? 1 : 0;
        if (!fc) build_site_lists(N, h.g2re.data(), h.h2_active, qsv[k], lists[k], true);
        h.single_groups = (!fc && records_single_groups(lists[k])) ? 1 : 0;
        build_q64(qsv[k], q64[k]);
        std::vector<QuartetRec>().swap(qsv[k]);
        h.site_entries = (int64_t)lists[k].entries.size();
        h.exec_flops_lists = list_exec_flops(lists[k], N, fc, !fc);
    }

    const auto t_p3 = clk();
    // ---- concatenate and upload
    int64_t ent_total = 0, split_total = 0, q_total = 0, g2_total = 0, spin_off = 0, rep_off = 0, chunk_total = 0;
    int64_t nb_total = 0;
    s->sd.resize(n);
    for (int k = 0; k < n; k++) {
        SampleHost& h = s->hs[k];
        SampleDev& d = s->sd[k];
        d.N = h.N;
        d.R = h.R;
        d.h2_active = h.h2_active;
        d.variant = variant;
        d.fc_tiles = h.fc_tiles;
        d.single_groups = h.single_groups;
        d.spin_off = spin_off;
        d.rep_off = rep_off;
        d.split_off = split_total;
        d.q_off = q_total;
        d.nq = (int64_t)q64[k].size();
        d.g2_off = g2_total;
        d.pair_off = -1;
        d.nb_off = nb_total;
        nb_total += (int64_t)h.N * ((h.N + 31) / 32);
        uint64_t pk = h.cfg.seed + 7000;
        const uint64_t key = splitmix64(pk);
        d.pair_key0 = (uint32_t)key;
        d.pair_key1 = (uint32_t)(key >> 32);
        spin_off += (int64_t)h.N * h.R;
        rep_off += h.R;
        split_total += (int64_t)h.N * (kSplit + 1);
        q_total += d.nq;
        g2_total += (int64_t)h.N * h.N;
        ent_total += h.site_entries;
        chunk_total += (int64_t)lists[k].chunk_start.size();
    }
    if (chunk_total >= (1ll << 31)) return bail(fail(PSPIN_ERR_ARG, "too many list chunks"));
    std::vector<int2> ent(ent_total);
    std::vector<int> site_chunks(split_total);
    std::vector<int64_t> chunk_start(chunk_total + 1);
    std::vector<Q64> qall(q_total);
    std::vector<uint32_t> nball(nb_total, 0u);
    std::vector<double> g2all(g2_total);
    std::vector<double> Eall(s->R_tot, 0.0);
    std::vector<uint64_t> kall(s->R_tot);
    {
        int64_t eoff = 0, coff = 0;
        for (int k = 0; k < n; k++) {
            const SampleDev& d = s->sd[k];
            std::copy(lists[k].entries.begin(), lists[k].entries.end(), ent.begin() + eoff);
            for (size_t t = 0; t < lists[k].chunk_start.size(); t++) chunk_start[coff + t] = lists[k].chunk_start[t] + eoff;
            for (size_t t = 0; t < lists[k].site_chunks.size(); t++)
                site_chunks[d.split_off + t] = (int)(lists[k].site_chunks[t] + coff);
            eoff += (int64_t)lists[k].entries.size();
            coff += (int64_t)lists[k].chunk_start.size();
            std::copy(q64[k].begin(), q64[k].end(), qall.begin() + d.q_off);
            {   // neighbour masks: sites that share an active quartet, or any g2 term, with m
                const int Nk = d.N, wpr = (Nk + 31) / 32;
                uint32_t* rows = nball.data() + d.nb_off;
                auto set = [&](int a, int b) { rows[(size_t)a * wpr + b / 32] |= 1u << (b % 32); };
                for (const Q64& q : q64[k]) {
                    const int v[4] = {q.i, q.j, q.k, q.lch & 0x3FFF};
                    for (int a = 0; a < 4; a++)
                        for (int b = 0; b < 4; b++)
                            if (a != b) set(v[a], v[b]);
                }
                if (d.h2_active)
                    for (int a = 0; a < Nk; a++)
                        for (int b = 0; b < Nk; b++)
                            if (a != b) set(a, b);
            }
            std::copy(s->hs[k].g2re.begin(), s->hs[k].g2re.end(), g2all.begin() + d.g2_off);
            std::copy(keys[k].begin(), keys[k].end(), kall.begin() + d.rep_off);
            lists[k] = SiteLists();
            q64[k].clear();
        }
        chunk_start[chunk_total] = eoff;
    }
    s->ent_total = ent_total;
    s->chunk_total = chunk_total;
    // units: replica blocks of 32, heaviest samples first
    for (int k = 0; k < n; k++)
        for (int rb = 0; rb < s->hs[k].R; rb += kRepBlock)
            s->units.push_back(Unit{k, rb, std::min(kRepBlock, s->hs[k].R - rb), 0});
    for (int K = 2; K <= 3; K++)
        for (int k = 0; k < n; k++)
            for (int rb = 0; rb < s->hs[k].R; rb += K * kRepBlock)
                s->units_k[K - 2].push_back(Unit{k, rb, std::min(K * kRepBlock, s->hs[k].R - rb), 0});
    for (std::vector<Unit>* u : {&s->units, &s->units_k[0], &s->units_k[1]})
        std::stable_sort(u->begin(), u->end(), [&](const Unit& a, const Unit& b) {
            return s->hs[a.sample].site_entries > s->hs[b.sample].site_entries;
        });
    if (s->opt.replicas_per_lane < 0 || s->opt.replicas_per_lane > 3)
        return bail(fail(PSPIN_ERR_ARG, "replicas_per_lane must be 0, 1, 2 or 3"));
    s->rpl = std::max(1, s->opt.replicas_per_lane);
    s->warps = choose_warps(s);
    if (s->warps < 0) return bail(fail(PSPIN_ERR_ARG, "warps_per_unit must be 1, 2, 4 or 8"));
    if (s->opt.wait_limit_clocks < 0 || s->opt.test_stall_move < 0)
        return bail(fail(PSPIN_ERR_ARG, "wait_limit_clocks and test_stall_move must be >= 0"));
    for (const SampleHost& h : s->hs) s->max_site_entries = std::max<int64_t>(s->max_site_entries, h.site_entries);
    {
        const int c = s->opt.cluster_size == 0 ? 1 : s->opt.cluster_size;
        s->warps2 = s->warps;
        if (c == -1) {
            const int rw = s->opt.warps_per_unit > 0 ? s->opt.warps_per_unit : 1;
            if (resident_smem_bytes_host(s->max_N, s->max_site_entries, rw) > 227 * 1024)
                return bail(fail(PSPIN_ERR_ARG, "the site lists do not fit in shared memory (cluster_size -1)"));
            s->cluster = 0;
            s->warps = rw;
        } else {
            if (c != 1 && c != 2 && c != 4 && c != 8 && c != 16)
                return bail(fail(PSPIN_ERR_ARG, "cluster_size must be -1, 1, 2, 4, 8 or 16"));
            if (c * s->warps > kSplit) return bail(fail(PSPIN_ERR_ARG, "cluster_size * warps_per_unit must be <= 32"));
            s->cluster = c;
            s->cluster2 = c;
        }
    }
    if (sweep_smem_bytes(s->max_N, s->warps) > 227 * 1024)
        return bail(fail(PSPIN_ERR_ARG, "N=%d needs more shared memory than a CTA has", s->max_N));
    if (s->rpl > 1 && s->cluster >= 1 && multi_smem_bytes_host(s->max_N, s->warps, s->cluster, s->rpl) > 227 * 1024)
        return bail(fail(PSPIN_ERR_ARG, "N=%d with %d replicas per lane needs more shared memory than a CTA has",
                         s->max_N, s->rpl));

    if ((rc = dalloc(&s->d_samples, n)) || (rc = dalloc(&s->d_units, s->units.size())) ||
        (rc = dalloc(&s->d_spins, (size_t)s->spin_total)) || (rc = dalloc(&s->d_E, s->R_tot)) ||
        (rc = dalloc(&s->d_beta, s->R_tot)) || (rc = dalloc(&s->d_target, s->R_tot)) ||
        (rc = dalloc(&s->d_drift, s->R_tot)) || (rc = dalloc(&s->d_e2, s->R_tot)) ||
        (rc = dalloc(&s->d_e4, s->R_tot)) || (rc = dalloc(&s->d_acc, s->R_tot)) ||
        (rc = dalloc(&s->d_prop, s->R_tot)) || (rc = dalloc(&s->d_key, s->R_tot)) ||
        (rc = dalloc(&s->d_entries, (size_t)ent_total)) || (rc = dalloc(&s->d_site_chunks, (size_t)split_total)) ||
        (rc = dalloc(&s->d_chunk_start, (size_t)chunk_total + 1)) ||
        (rc = dalloc(&s->d_q64, (size_t)std::max<int64_t>(q_total, 1))) ||
        (rc = dalloc(&s->d_g2, (size_t)g2_total)) || (rc = dalloc(&s->d_sweep_counter, 1)) ||
        (rc = dalloc(&s->d_nbmask, (size_t)std::max<int64_t>(nb_total, 1))) ||
        (rc = dalloc(&s->d_status, 1)) || (rc = dalloc(&s->d_units_k[0], s->units_k[0].size())) ||
        (rc = dalloc(&s->d_units_k[1], s->units_k[1].size())))
        return bail(rc);
    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        if (!bytes) return PSPIN_OK;
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->st);
        if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
        return PSPIN_OK;
    };
    std::vector<double> ones(s->R_tot);
    for (int k = 0; k < n; k++)
        for (int r = 0; r < s->hs[k].R; r++) ones[s->sd[k].rep_off + r] = 1.0 / s->hs[k].cfg.T;
    if ((rc = up(s->d_samples, s->sd.data(), n * sizeof(SampleDev))) ||
        (rc = up(s->d_units, s->units.data(), s->units.size() * sizeof(Unit))) ||
        (rc = up(s->d_units_k[0], s->units_k[0].data(), s->units_k[0].size() * sizeof(Unit))) ||
        (rc = up(s->d_units_k[1], s->units_k[1].data(), s->units_k[1].size() * sizeof(Unit))) ||
        (rc = up(s->d_key, kall.data(), kall.size() * sizeof(uint64_t))) ||
        (rc = up(s->d_entries, ent.data(), ent.size() * sizeof(int2))) ||
        (rc = up(s->d_site_chunks, site_chunks.data(), site_chunks.size() * sizeof(int))) ||
        (rc = up(s->d_chunk_start, chunk_start.data(), chunk_start.size() * sizeof(int64_t))) ||
        (rc = up(s->d_q64, qall.data(), qall.size() * sizeof(Q64))) ||
        (rc = up(s->d_g2, g2all.data(), g2all.size() * sizeof(double))) ||
        (rc = up(s->d_nbmask, nball.data(), nball.size() * sizeof(uint32_t))) ||
        (rc = up(s->d_beta, ones.data(), ones.size() * sizeof(double))))
        return bail(rc);
    {
        cudaError_t e = cudaMemsetAsync(s->d_acc, 0, s->R_tot * sizeof(long long), s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_prop, 0, s->R_tot * sizeof(long long), s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_E, 0, s->R_tot * sizeof(double), s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_drift, 0, s->R_tot * sizeof(double), s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_sweep_counter, 0, sizeof(long long), s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_status, 0, sizeof(int), s->st);
        if (e != cudaSuccess) return bail(fail(PSPIN_ERR_CUDA, "memset: %s", cudaGetErrorString(e)));
    }
    if (s->opt.trace_replica >= 0 && s->opt.trace_capacity > 0) {
        if ((rc = dalloc(&s->d_trace, (size_t)s->opt.trace_capacity))) return bail(rc);
        cudaMemsetAsync(s->d_trace, 0, sizeof(pspin_move_record) * (size_t)s->opt.trace_capacity, s->st);
    }
    // replica amplitudes projected onto the constraint on the device, in the
    // reference's way (spins.cu:27-111, spins_sparse.cu:28-80), as FP32 in the
    // [site][replica] layout; each replica's constraint value as its target
    for (int k = 0; k < n; k++) {
        const SampleDev& d = s->sd[k];
        cudaError_t e = dev_normalize_replicas(nrm_dev.p[k], d.N, d.R, variant == PSPIN_SPARSE, s->opt.init_exact,
                                               s->d_spins + d.spin_off, s->d_target + d.rep_off, s->st);
        if (e != cudaSuccess) return bail(fail(PSPIN_ERR_CUDA, "spin normalisation: %s", cudaGetErrorString(e)));
    }
    // initial energies (the chain's form, FP64, from the FP32 amplitudes)
    if ((rc = run_energy(s, nullptr, nullptr, true, false))) return bail(rc);
    {
        cudaError_t e = cudaStreamSynchronize(s->st);
        if (e != cudaSuccess) return bail(fail(PSPIN_ERR_CUDA, "init: %s", cudaGetErrorString(e)));
    }
    if (timing)
        fprintf(stderr, "[pspin set-up] device phase %.3f s, host layout %.3f s, upload+energies %.3f s\n",
                secs(t_p1, t_p2), secs(t_p2, t_p3), secs(t_p3, clk()));
    *out = s;
    return PSPIN_OK;
}

extern "C" int pspin_create(const pspin_config* cfg, int variant, const pspin_options* opt, pspin_state** out) {
    return pspin_create_batch(cfg, 1, variant, opt, out);
}

extern "C" int pspin_destroy(pspin_state* s) {
    if (!s) return PSPIN_OK;
    cudaStreamSynchronize(s->st);
    free_state(s);
    return PSPIN_OK;
}

extern "C" int pspin_total_replicas(const pspin_state* s) { return s ? s->R_tot : 0; }
extern "C" int pspin_num_samples(const pspin_state* s) { return s ? s->S : 0; }

// ------------------------------------------------------------------ sweeps
// Enqueues one step: a sweep launch of nsweeps sweeps, the exchange launch
// (which advances the device sweep counter) and, after an exchange, the
// observable recorder.  No host bookkeeping, so a sequence of steps can be
// captured in a CUDA graph; e0/e1 (optional) bracket the sweep kernel.
static int enqueue_step(pspin_state* s, int nsweeps, bool exchange, cudaEvent_t e0, cudaEvent_t e1) {
    SweepParams p{};
    p.samples = s->d_samples;
    p.units = s->d_units;
    p.spins = s->d_spins;
    p.energy = s->d_E;
    p.accepted = s->d_acc;
    p.proposed = s->d_prop;
    p.beta = s->d_beta;
    p.key = s->d_key;
    p.entries = s->d_entries;
    p.chunk_start = s->d_chunk_start;
    p.site_chunks = s->d_site_chunks;
    p.pair_chunks = s->d_pair_chunks;
    p.site_chunks_g = s->d_site_chunks_g;
    p.nbmask = s->d_nbmask;
    p.sweep_counter = s->d_sweep_counter;
    p.nsweeps = nsweeps;
    p.warps = s->proposal == PSPIN_PROPOSAL_PLAIN ? s->warps : s->warps2;
    p.trace_sample = s->opt.trace_sample;
    p.trace_rep = s->opt.trace_replica;
    p.trace_cap = s->opt.trace_capacity;
    p.trace_sweep0 = s->trace_sweep0;
    p.trace = s->d_trace;
    p.status = s->d_status;
    p.wait_clocks = s->opt.wait_limit_clocks > 0 ? (long long)s->opt.wait_limit_clocks : kWaitClocks;
    p.stall_move = s->opt.test_stall_move > 0 ? s->opt.test_stall_move - 1 : -1;
    if (e0) CK(cudaEventRecord(e0, s->st));
    p.cluster = s->proposal == PSPIN_PROPOSAL_PLAIN ? s->cluster : s->cluster2;
    if (s->proposal == PSPIN_PROPOSAL_PLAIN && s->cluster == 0) {
        CK(launch_sweep_resident(p, (int)s->units.size(), s->variant, s->max_N, s->max_site_entries, s->st));
    } else if (s->proposal == PSPIN_PROPOSAL_PLAIN && s->rpl > 1) {
        const std::vector<Unit>& u = s->units_k[s->rpl - 2];
        p.units = s->d_units_k[s->rpl - 2];
        CK(launch_sweep_multi(p, (int)u.size(), s->variant, s->max_N, s->rpl, s->st, nullptr));
    } else if (s->proposal == PSPIN_PROPOSAL_PLAIN && s->cluster > 1) {
        CK(launch_sweep_cluster(p, (int)s->units.size(), s->variant, s->max_N, s->st, nullptr));
    } else if (s->proposal == PSPIN_PROPOSAL_PLAIN) {
        CK(launch_sweep(p, (int)s->units.size(), s->variant, s->max_N, s->st));
    } else {
        if (!s->d_site_chunks_g || !s->d_pair_chunks)
            return fail(PSPIN_ERR_STATE, "two-pass sweep without its group-format lists (pspin_set_proposal builds them)");
        LearnParams lp{};
        lp.mode = s->proposal;
        lp.w = s->d_wbf;
        lp.records = s->d_records;
        lp.rec_count = s->d_rec_count;
        lp.rec_cap = s->rec_cap;
        lp.rec_prob = s->rec_prob;
        CK(launch_learned_sweep(p, lp, (int)s->units.size(), s->max_N, s->st, nullptr));
    }
    if (e1) CK(cudaEventRecord(e1, s->st));
    ExchangeParams x{};
    x.n_samples = s->S;
    x.NT = s->pt_NT;
    x.nrep = s->pt_nrep;
    x.samples = s->d_samples;
    x.beta_sched = s->d_beta_sched;
    x.energy = s->d_E;
    x.beta = s->d_beta;
    x.perm = s->d_perm;
    x.drand_state = s->d_drand;
    x.ex_acc = s->d_ex_acc;
    x.ex_prop = s->d_ex_prop;
    x.sweep_counter = s->d_sweep_counter;
    x.nsweeps_done = nsweeps;
    x.do_exchange = exchange ? 1 : 0;
    CK(launch_exchange(x, s->st));
    if (exchange && s->obs_cap > 0) {
        ObserveParams o{};
        o.n_samples = s->S;
        o.NT = s->pt_NT;
        o.nrep = s->pt_nrep;
        o.temp_index = s->obs_t;
        o.capacity = s->obs_cap;
        o.pt_freq = s->pt_freq;
        o.samples = s->d_samples;
        o.spins = s->d_spins;
        o.energy = s->d_E;
        o.perm = s->d_perm;
        o.sweep_counter = s->d_sweep_counter;
        o.sweep0 = s->obs_sweep0;
        o.E_out = s->d_obs_E;
        o.q_out = s->d_obs_q;
        CK(launch_observe(o, s->st));
    }
    return PSPIN_OK;
}

static int do_resync(pspin_state* s);

// host counters after `steps` steps of nsweeps sweeps each; the resync when due
static int account_steps(pspin_state* s, int steps, int nsweeps, bool exchange) {
    s->sweep_launches += steps;
    s->kernel_launches += (long long)steps * (2 + ((exchange && s->obs_cap > 0) ? 1 : 0));
    s->sweeps_done += (long long)steps * nsweeps;
    s->since_resync += (long long)steps * nsweeps;
    if (s->opt.resync_every > 0 && s->since_resync >= s->opt.resync_every) {
        TRY(do_resync(s));
        s->since_resync = 0;
    }
    return PSPIN_OK;
}

static int launch_chunk(pspin_state* s, int nsweeps, bool exchange) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (s->profiling) {
        if (s->ev_used == s->ev_pool.size()) {
            std::pair<cudaEvent_t, cudaEvent_t> pr;
            CK(cudaEventCreate(&pr.first));
            CK(cudaEventCreate(&pr.second));
            s->ev_pool.push_back(pr);
        }
        e0 = s->ev_pool[s->ev_used].first;
        e1 = s->ev_pool[s->ev_used].second;
        s->ev_used++;
    }
    TRY(enqueue_step(s, nsweeps, exchange, e0, e1));
    return account_steps(s, 1, nsweeps, exchange);
}

static void drop_graph(pspin_state* s) {
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    s->graph_exec = nullptr;
}

static int graph_steps(const pspin_state* s) {
    const int g = s->opt.graph_steps;
    return g == 0 ? 32 : (g < 0 ? 0 : g);
}

// One graph of G PT steps (pt_freq sweeps, exchange, observe), captured on
// the engine's stream.  The kernels read the sweep index from the device
// counter that the exchange kernel advances, so every replay continues the
// same move and pair streams as direct launches would.
static int capture_graph(pspin_state* s, int G) {
    drop_graph(s);
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    int rc = PSPIN_OK;
    for (int g = 0; g < G && rc == PSPIN_OK; g++) rc = enqueue_step(s, s->pt_freq, true, nullptr, nullptr);
    cudaError_t e = cudaStreamEndCapture(s->st, &graph);
    if (rc != PSPIN_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&s->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        s->graph_exec = nullptr;
        return fail(PSPIN_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    s->graph_G = G;
    return PSPIN_OK;
}

static int timeout_error(int status) {
    return fail(PSPIN_ERR_TIMEOUT,
                "a bounded wait in the sweep kernel ran out (status %d%s): the replica blocks whose wait ran out "
                "abandoned that launch and kept their state from before it",
                status, (status & kStatusDrain) ? ", and the drain of its copies ran out too" : "");
}

static int run_sweeps(pspin_state* s, int nsweeps, bool pt) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (nsweeps < 0) return fail(PSPIN_ERR_ARG, "nsweeps < 0");
    const int G = (pt && !s->profiling) ? graph_steps(s) : 0;
    CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->st));   // a time-out is reported by the call it happens in
    int left = nsweeps;
    while (left > 0) {
        // whole graphs of G steps up to the next resync, from a step boundary
        if (G > 0 && s->sweeps_done % s->pt_freq == 0) {
            long long room = left;
            if (s->opt.resync_every > 0) room = std::min<long long>(room, s->opt.resync_every - s->since_resync);
            const long long reps = room / ((long long)G * s->pt_freq);
            if (reps > 0) {
                if (!s->graph_exec || s->graph_G != G) TRY(capture_graph(s, G));
                for (long long r = 0; r < reps; r++) {
                    CK(cudaGraphLaunch(s->graph_exec, s->st));
                    s->graph_launches++;
                    TRY(account_steps(s, G, s->pt_freq, true));
                }
                left -= (int)(reps * G * s->pt_freq);
                continue;
            }
        }
        int chunk = left;
        if (s->opt.resync_every > 0) chunk = std::min<long long>(chunk, s->opt.resync_every - s->since_resync);
        bool ex = false;
        if (pt) {
            const int to_ex = s->pt_freq - (int)(s->sweeps_done % s->pt_freq);
            if (to_ex <= chunk) {
                chunk = to_ex;
                ex = true;
            }
        }
        if (chunk <= 0) chunk = 1;
        TRY(launch_chunk(s, chunk, ex));
        left -= chunk;
    }
    CK(cudaStreamSynchronize(s->st));
    int status = 0;
    CK(cudaMemcpy(&status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status) return timeout_error(status);
    return PSPIN_OK;
}

// Whether `cluster` CTAs of `warps` warps can hold one replica block (shared
// memory, co-residency of the cluster); the plain kernel for cluster 1.
static bool shape_fits(pspin_state* s, int warps, int cluster, int K = 1) {
    if (cluster == 0)
        return K == 1 && s->proposal == PSPIN_PROPOSAL_PLAIN &&
               resident_smem_bytes_host(s->max_N, s->max_site_entries, warps) <= 227 * 1024;
    if (cluster * warps > kSplit) return false;
    if (K > 1) {
        if (s->proposal != PSPIN_PROPOSAL_PLAIN) return false;
        if (multi_smem_bytes_host(s->max_N, warps, cluster, K) > 227 * 1024) return false;
        SweepParams p{};
        p.warps = warps;
        p.cluster = cluster;
        int n = 0;
        if (launch_sweep_multi(p, (int)s->units_k[K - 2].size(), s->variant, s->max_N, K, s->st, &n) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return n > 0;
    }
    if (s->proposal != PSPIN_PROPOSAL_PLAIN) {
        if (learned_smem_bytes_host(s->max_N, warps, cluster) > 227 * 1024) return false;
        if (cluster == 1) return true;
        SweepParams p{};
        p.warps = warps;
        p.cluster = cluster;
        LearnParams lp{};
        int n = 0;
        if (launch_learned_sweep(p, lp, (int)s->units.size(), s->max_N, s->st, &n) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return n > 0;
    }
    if (cluster == 1) return sweep_smem_bytes(s->max_N, warps) <= 227 * 1024;
    if (cluster_smem_bytes_host(s->max_N, warps, cluster) > 227 * 1024) return false;
    SweepParams p{};
    p.warps = warps;
    p.cluster = cluster;
    int n = 0;
    if (launch_sweep_cluster(p, (int)s->units.size(), s->variant, s->max_N, s->st, &n) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n > 0;
}

// Times `sweeps` sweeps (no exchange) for every block shape -- CTAs per
// replica block (cluster) x warps per CTA -- from the same saved state and
// keeps the fastest.  The state (amplitudes, energies, counters, sweep index)
// is restored after every trial, so the chain continues as if the trials had
// not run.
static int autotune(pspin_state* s, int sweeps, int k_lo, int k_hi, int* chosen_warps, int* chosen_cluster,
                    int* chosen_k, float* ms_out) {
    if (!s || sweeps < 1) return fail(PSPIN_ERR_ARG, "bad arguments");
    float2* b_spins = nullptr;
    double* b_E = nullptr;
    long long *b_acc = nullptr, *b_prop = nullptr, *b_cnt = nullptr;
    int rc;
    if ((rc = dalloc(&b_spins, (size_t)s->spin_total)) || (rc = dalloc(&b_E, s->R_tot)) ||
        (rc = dalloc(&b_acc, s->R_tot)) || (rc = dalloc(&b_prop, s->R_tot)) || (rc = dalloc(&b_cnt, 1))) {
        cudaFree(b_spins); cudaFree(b_E); cudaFree(b_acc); cudaFree(b_prop); cudaFree(b_cnt);
        return rc;
    }
    auto copy_all = [&](bool save) -> cudaError_t {
        const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
        struct { void* a; void* b; size_t n; } t[] = {
            {b_spins, s->d_spins, s->spin_total * sizeof(float2)}, {b_E, s->d_E, s->R_tot * sizeof(double)},
            {b_acc, s->d_acc, s->R_tot * sizeof(long long)}, {b_prop, s->d_prop, s->R_tot * sizeof(long long)},
            {b_cnt, s->d_sweep_counter, sizeof(long long)}};
        for (auto& c : t) {
            cudaError_t e = save ? cudaMemcpyAsync(c.a, c.b, c.n, k, s->st) : cudaMemcpyAsync(c.b, c.a, c.n, k, s->st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    const bool plain = s->proposal == PSPIN_PROPOSAL_PLAIN;
    int& W = plain ? s->warps : s->warps2;   // the current proposal's kernel is tuned
    int& Cl = plain ? s->cluster : s->cluster2;
    const int w0 = W, c0 = Cl, k0 = s->rpl;
    const float prob0 = s->rec_prob;
    s->rec_prob = 0.f;                       // trials record no training moves
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaError_t e = cudaMemsetAsync(s->d_status, 0, sizeof(int), s->st);
    if (e == cudaSuccess) e = copy_all(true);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    int best_w = w0, best_c = c0, best_k = k0;
    float best_ms = 0.f;
    const int cw[4] = {1, 2, 4, 8}, cc[6] = {0, 1, 2, 4, 8, 16};
    for (int K = k_lo; K <= k_hi; K++)
    for (int ci = 0; ci < 6; ci++)
        for (int wi = 0; wi < 4; wi++) {
            float ms = -1.f;
            if (e == cudaSuccess && rc == PSPIN_OK && shape_fits(s, cw[wi], cc[ci], K)) {
                W = cw[wi];
                Cl = cc[ci];
                if (plain) s->rpl = K;
                rc = enqueue_step(s, 1, false, nullptr, nullptr);          // warm-up sweep
                if (rc == PSPIN_OK) e = cudaEventRecord(t0, s->st);
                for (int k = 0; k < sweeps && rc == PSPIN_OK && e == cudaSuccess; k++)
                    rc = enqueue_step(s, 1, false, nullptr, nullptr);
                if (rc == PSPIN_OK && e == cudaSuccess) e = cudaEventRecord(t1, s->st);
                if (rc == PSPIN_OK && e == cudaSuccess) e = cudaEventSynchronize(t1);
                if (rc == PSPIN_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
                if (rc == PSPIN_OK && e == cudaSuccess) {
                    ms /= sweeps;
                    if (best_ms <= 0.f || ms < best_ms) {
                        best_ms = ms;
                        best_w = cw[wi];
                        best_c = cc[ci];
                        best_k = K;
                    }
                }
                if (e == cudaSuccess) e = copy_all(false);
            }
            if (ms_out) ms_out[((K - k_lo) * 6 + ci) * 4 + wi] = ms;
        }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    int status = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(b_spins); cudaFree(b_E); cudaFree(b_acc); cudaFree(b_prop); cudaFree(b_cnt);
    s->rec_prob = prob0;
    const bool good = rc == PSPIN_OK && e == cudaSuccess;
    W = good ? best_w : w0;
    Cl = good ? best_c : c0;
    if (plain) s->rpl = good ? best_k : k0;
    drop_graph(s);
    if (rc != PSPIN_OK) return rc;
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    if (status) return timeout_error(status);
    if (chosen_warps) *chosen_warps = W;
    if (chosen_cluster) *chosen_cluster = Cl;
    if (chosen_k) *chosen_k = plain ? s->rpl : 1;
    return PSPIN_OK;
}

extern "C" int pspin_autotune(pspin_state* s, int sweeps, int* chosen_warps, int* chosen_cluster, float* ms_out) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    const int K = s->proposal == PSPIN_PROPOSAL_PLAIN ? s->rpl : 1;
    return autotune(s, sweeps, K, K, chosen_warps, chosen_cluster, nullptr, ms_out);
}

extern "C" int pspin_autotune_lanes(pspin_state* s, int sweeps, int* chosen_warps, int* chosen_cluster,
                                    int* chosen_replicas_per_lane, float* ms_out) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (s->proposal != PSPIN_PROPOSAL_PLAIN)
        return fail(PSPIN_ERR_ARG, "pspin_autotune_lanes tunes the plain sweep (use pspin_autotune)");
    return autotune(s, sweeps, 1, 3, chosen_warps, chosen_cluster, chosen_replicas_per_lane, ms_out);
}

extern "C" int pspin_sweep(pspin_state* s, int nsweeps) { return run_sweeps(s, nsweeps, false); }

extern "C" int pspin_set_betas(pspin_state* s, const double* betas) {
    if (!s || !betas) return fail(PSPIN_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(s->d_beta, betas, s->R_tot * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_fill_betas(pspin_state* s, double beta) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    std::vector<double> b(s->R_tot, beta);
    return pspin_set_betas(s, b.data());
}

extern "C" int pspin_get_results(pspin_state* s, double* E, int64_t* acc, int64_t* prop) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (E) CK(cudaMemcpyAsync(E, s->d_E, s->R_tot * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    if (acc) CK(cudaMemcpyAsync(acc, s->d_acc, s->R_tot * sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    if (prop) CK(cudaMemcpyAsync(prop, s->d_prop, s->R_tot * sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_reset_counters(pspin_state* s) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    CK(cudaMemsetAsync(s->d_acc, 0, s->R_tot * sizeof(long long), s->st));
    CK(cudaMemsetAsync(s->d_prop, 0, s->R_tot * sizeof(long long), s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_get_spins(pspin_state* s, double* out) {
    if (!s || !out) return fail(PSPIN_ERR_ARG, "null argument");
    std::vector<float2> h(s->spin_total);
    CK(cudaMemcpyAsync(h.data(), s->d_spins, h.size() * sizeof(float2), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int k = 0; k < s->S; k++) {
        const SampleDev& d = s->sd[k];
        for (int r = 0; r < d.R; r++)
            for (int i = 0; i < d.N; i++) {
                const float2 v = h[d.spin_off + (int64_t)i * d.R + r];
                double* o = out + 2 * ((int64_t)d.N * (d.rep_off + r) - (int64_t)d.N * d.rep_off + d.spin_off) + 2 * i;
                o[0] = v.x;
                o[1] = v.y;
            }
    }
    return PSPIN_OK;
}

extern "C" int pspin_set_spins(pspin_state* s, const double* in) {
    if (!s || !in) return fail(PSPIN_ERR_ARG, "null argument");
    std::vector<float2> h(s->spin_total);
    for (int k = 0; k < s->S; k++) {
        const SampleDev& d = s->sd[k];
        for (int r = 0; r < d.R; r++)
            for (int i = 0; i < d.N; i++) {
                const double* o = in + 2 * (d.spin_off + (int64_t)d.N * r) + 2 * i;
                h[d.spin_off + (int64_t)i * d.R + r] = make_float2((float)o[0], (float)o[1]);
            }
    }
    CK(cudaMemcpyAsync(s->d_spins, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice, s->st));
    TRY(run_energy(s, nullptr, nullptr, true, false));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_split_energies(pspin_state* s, double* e2, double* e4) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    TRY(run_energy(s, s->d_e2, s->d_e4, false, false));
    if (e2) CK(cudaMemcpyAsync(e2, s->d_e2, s->R_tot * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    if (e4) CK(cudaMemcpyAsync(e4, s->d_e4, s->R_tot * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_resync(pspin_state* s) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    TRY(run_energy(s, nullptr, nullptr, true, true));
    s->since_resync = 0;
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

// ------------------------------------------------------------------ introspection
extern "C" int pspin_get_info(pspin_state* s, int sample, pspin_info* info) {
    if (!s || !info || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    const SampleHost& h = s->hs[sample];
    info->N = h.N;
    info->nrep = h.R;
    info->h2_active = h.h2_active;
    info->n_quartets = (int)(h.sqg.size());
    info->n_pairs_active = h.n_pairs_active;
    info->n_quart_active = h.n_quart_active;
    info->site_entries = h.site_entries;
    return PSPIN_OK;
}

// Work of one sweep of every sample and replica.  Algorithmic: the
// reference's per-move operation count F = 20 W4 + 4 W2 + 64 (a quartet term
// as a 4-factor complex product times the coupling plus the accumulate, an
// H2 term as one complex FMA pair, 64 for proposal and decision) with
// W4 = A (8/N - 12/(N(N-1))) and W2 = P (4/N - 2/(N(N-1))) the expected
// active quartets and off-diagonal pairs touching a uniformly random pair
// (A = active quartet-channel pairs, P = active off-diagonal g2 pairs).
// Executed: what the field kernels run -- per replica the operations of
// accumulating the lists of the move's two sites (14 per group header and 4
// per data entry; 56 per tile header and 16 per tile row), whose expectation
// over a sweep's N/2 uniformly random pairs is one pass over all N lists,
// plus the same 64 per move for proposal and decision.
extern "C" int pspin_sweep_work(pspin_state* s, double* algorithmic_flops, double* executed_flops) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    double alg = 0.0, ex = 0.0;
    for (const SampleHost& h : s->hs) {
        const double N = h.N, R = h.R, moves = R * (double)(h.N / 2);
        // active quartet-channel pairs: the mask's survivors (dense) or the
        // selected quartets (sparse)
        const double A = s->variant == PSPIN_SPARSE ? (double)h.sqg.size() : (double)h.n_quart_active;
        const double P = h.h2_active ? (double)(h.n_pairs_active - h.N) : 0.0;   // the count includes the diagonal
        const double W4 = A * (8.0 / N - 12.0 / (N * (N - 1.0)));
        const double W2 = P * (4.0 / N - 2.0 / (N * (N - 1.0)));
        alg += moves * (20.0 * W4 + 4.0 * W2 + 64.0);
        ex += R * h.exec_flops_lists + moves * 64.0;
    }
    if (algorithmic_flops) *algorithmic_flops = alg;
    if (executed_flops) *executed_flops = ex;
    return PSPIN_OK;
}

extern "C" int pspin_device_arrays(pspin_state* s, int64_t** accepted, int64_t** proposed, double** energies,
                                   double** betas) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    static_assert(sizeof(long long) == sizeof(int64_t), "counter width");
    if (accepted) *accepted = reinterpret_cast<int64_t*>(s->d_acc);
    if (proposed) *proposed = reinterpret_cast<int64_t*>(s->d_prop);
    if (energies) *energies = s->d_E;
    if (betas) *betas = s->d_beta;
    return PSPIN_OK;
}

extern "C" int pspin_get_omega(pspin_state* s, int sample, double* omega) {
    if (!s || !omega || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    const SampleHost& h = s->hs[sample];
    if (h.omega.empty()) return fail(PSPIN_ERR_STATE, "fully connected sample has no frequencies");
    std::copy(h.omega.begin(), h.omega.end(), omega);
    return PSPIN_OK;
}

extern "C" int pspin_get_couplings(pspin_state* s, int sample, double* g2, double* g4, uint8_t* mask) {
    if (!s || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    const SampleHost& h = s->hs[sample];
    if (g2)
        for (size_t t = 0; t < h.g2re.size(); t++) { g2[2 * t] = h.g2re[t]; g2[2 * t + 1] = 0.0; }
    if (g4 || mask) {
        if (s->variant != PSPIN_DENSE) return fail(PSPIN_ERR_STATE, "sparse variant keeps no dense g4");
        if (g4) {
            std::vector<double> t(h.nq_dense);
            CK(cudaMemcpyAsync(t.data(), s->d_g4re + h.g4_off, h.nq_dense * sizeof(double), cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            for (int64_t q = 0; q < h.nq_dense; q++) { g4[2 * q] = t[q]; g4[2 * q + 1] = 0.0; }
        }
        if (mask) {
            CK(cudaMemcpyAsync(mask, s->d_mask + h.g4_off, h.nq_dense, cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
        }
    }
    return PSPIN_OK;
}

extern "C" int pspin_get_sparse_quartets(pspin_state* s, int sample, int32_t* ijklch, double* g) {
    if (!s || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    const SampleHost& h = s->hs[sample];
    if (s->variant != PSPIN_SPARSE) return fail(PSPIN_ERR_STATE, "dense variant has no sparse quartet list");
    if (ijklch) std::copy(h.sq.begin(), h.sq.end(), ijklch);
    if (g) std::copy(h.sqg.begin(), h.sqg.end(), g);
    return PSPIN_OK;
}

// ------------------------------------------------------------------ parallel tempering
extern "C" int pspin_pt_init(pspin_state* s, int NT, int nrep, const double* beta_sched, int pt_freq) {
    if (!s || !beta_sched) return fail(PSPIN_ERR_ARG, "null argument");
    if (NT < 2 || nrep < 1 || pt_freq < 1) return fail(PSPIN_ERR_ARG, "need NT >= 2, nrep >= 1, pt_freq >= 1");
    drop_graph(s);
    for (const SampleHost& h : s->hs)
        if (h.R != NT * nrep) return fail(PSPIN_ERR_ARG, "sample nrep %d != NT*nrep_per_temp %d", h.R, NT * nrep);
    cudaFree(s->d_beta_sched);
    cudaFree(s->d_perm);
    cudaFree(s->d_drand);
    cudaFree(s->d_ex_acc);
    cudaFree(s->d_ex_prop);
    s->d_beta_sched = nullptr; s->d_perm = nullptr; s->d_drand = nullptr; s->d_ex_acc = nullptr; s->d_ex_prop = nullptr;
    s->pt_NT = NT;
    s->pt_nrep = nrep;
    s->pt_freq = pt_freq;
    int rc;
    if ((rc = dalloc(&s->d_beta_sched, NT)) || (rc = dalloc(&s->d_perm, (size_t)s->S * NT * nrep)) ||
        (rc = dalloc(&s->d_drand, s->S)) || (rc = dalloc(&s->d_ex_acc, (size_t)s->S * (NT - 1))) ||
        (rc = dalloc(&s->d_ex_prop, (size_t)s->S * (NT - 1))))
        return rc;
    std::vector<int> perm((size_t)s->S * NT * nrep);
    std::vector<unsigned long long> dr(s->S);
    std::vector<double> betas(s->R_tot);
    for (int k = 0; k < s->S; k++) {
        for (int i = 0; i < NT * nrep; i++) perm[(size_t)k * NT * nrep + i] = i;   // :283-284
        dr[k] = srand48_state((long)s->hs[k].cfg.seed + 5000);                        // :304
        for (int t = 0; t < NT; t++)
            for (int r = 0; r < nrep; r++) betas[s->sd[k].rep_off + t * nrep + r] = beta_sched[t];  // :274-278
    }
    CK(cudaMemcpyAsync(s->d_beta_sched, beta_sched, NT * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_drand, dr.data(), dr.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->d_ex_acc, 0, (size_t)s->S * (NT - 1) * sizeof(long long), s->st));
    CK(cudaMemsetAsync(s->d_ex_prop, 0, (size_t)s->S * (NT - 1) * sizeof(long long), s->st));
    CK(cudaMemcpyAsync(s->d_beta, betas.data(), betas.size() * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_pt_run(pspin_state* s, int nsweeps) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (s->pt_NT < 2) return fail(PSPIN_ERR_STATE, "pspin_pt_init has not been called");
    return run_sweeps(s, nsweeps, true);
}

extern "C" int pspin_pt_get(pspin_state* s, int sample, int32_t* perm, int64_t* ex_acc, int64_t* ex_prop) {
    if (!s || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    if (s->pt_NT < 2) return fail(PSPIN_ERR_STATE, "pspin_pt_init has not been called");
    const int NT = s->pt_NT, nr = s->pt_nrep;
    if (perm) CK(cudaMemcpyAsync(perm, s->d_perm + (size_t)sample * NT * nr, NT * nr * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    if (ex_acc) CK(cudaMemcpyAsync(ex_acc, s->d_ex_acc + (size_t)sample * (NT - 1), (NT - 1) * sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    if (ex_prop) CK(cudaMemcpyAsync(ex_prop, s->d_ex_prop + (size_t)sample * (NT - 1), (NT - 1) * sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_observe_init(pspin_state* s, int temp_index, int capacity) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (s->pt_NT < 2) return fail(PSPIN_ERR_STATE, "pspin_pt_init has not been called");
    if (temp_index < 0 || temp_index >= s->pt_NT || capacity < 0)
        return fail(PSPIN_ERR_ARG, "temperature index %d outside [0, %d) or negative capacity", temp_index, s->pt_NT);
    drop_graph(s);
    cudaFree(s->d_obs_E);
    cudaFree(s->d_obs_q);
    s->d_obs_E = nullptr;
    s->d_obs_q = nullptr;
    s->obs_cap = 0;
    if (capacity == 0) return PSPIN_OK;
    const int nr = s->pt_nrep, npairs = nr * (nr - 1) / 2;
    int rc;
    if ((rc = dalloc(&s->d_obs_E, (size_t)capacity * s->S * nr)) ||
        (rc = dalloc(&s->d_obs_q, (size_t)capacity * s->S * std::max(npairs, 1))))
        return rc;
    CK(cudaMemcpyAsync(&s->obs_sweep0, s->d_sweep_counter, sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->obs_t = temp_index;
    s->obs_cap = capacity;
    return PSPIN_OK;
}

extern "C" int pspin_observe_get(pspin_state* s, int64_t* n_rows, double* energy, double* overlap, int max_rows) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (s->obs_cap <= 0) return fail(PSPIN_ERR_STATE, "pspin_observe_init has not been called");
    long long counter = 0;
    CK(cudaMemcpyAsync(&counter, s->d_sweep_counter, sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    long long n = (counter - s->obs_sweep0) / s->pt_freq;
    n = std::max(0LL, std::min<long long>(n, s->obs_cap));
    if (n_rows) *n_rows = n;
    const long long m = std::min<long long>(n, std::max(max_rows, 0));
    const int nr = s->pt_nrep, npairs = nr * (nr - 1) / 2;
    if (energy && m > 0)
        CK(cudaMemcpyAsync(energy, s->d_obs_E, (size_t)m * s->S * nr * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    if (overlap && m > 0 && npairs > 0)
        CK(cudaMemcpyAsync(overlap, s->d_obs_q, (size_t)m * s->S * npairs * sizeof(double), cudaMemcpyDeviceToHost,
                           s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

// Host-side exchange for drivers that keep the PT loop on the host, as the
// reference's driver does (parallel_tempering.cu:316-352): t from the hottest
// pair up, a swap applied before the next t, drand48 drawn only when delta < 0,
// then betas rebuilt from perm (:347-351).  Samples are independent (OpenMP).
extern "C" int pspin_overlap_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                         double qmin, double qmax, long long* counts, const char** err);

extern "C" int pspin_overlap_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, double qmin,
                                    double qmax, int64_t* counts) {
    const char* err = nullptr;
    const int rc = pspin_overlap_counts_impl(N, NT, nrep, nsnap, configs, nbins, qmin, qmax,
                                             reinterpret_cast<long long*>(counts), &err);
    if (rc == 1) return fail(PSPIN_ERR_ARG, "%s", err);
    if (rc) return fail(PSPIN_ERR_CUDA, "overlap counts: %s", err);
    return PSPIN_OK;
}

extern "C" int pspin_ifo_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                     double cmin, double cmax, long long* ifo_counts, long long* ifo_n,
                                     long long* exp_counts, long long* exp_n, const char** err);

extern "C" int pspin_ifo_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, double cmin,
                                double cmax, int64_t* ifo_counts, int64_t* ifo_n, int64_t* exp_counts,
                                int64_t* exp_n) {
    const char* err = nullptr;
    const int rc = pspin_ifo_counts_impl(N, NT, nrep, nsnap, configs, nbins, cmin, cmax,
                                         reinterpret_cast<long long*>(ifo_counts), reinterpret_cast<long long*>(ifo_n),
                                         reinterpret_cast<long long*>(exp_counts), reinterpret_cast<long long*>(exp_n),
                                         &err);
    if (rc == 1) return fail(PSPIN_ERR_ARG, "%s", err);
    if (rc) return fail(PSPIN_ERR_CUDA, "IFO counts: %s", err);
    return PSPIN_OK;
}

extern "C" int pspin_deeper_counts_impl(int N, int NT, int nrep, int nsnap, const double* configs, int nbins,
                                        int nbins_a2, double da2, const int32_t* quartets, int M, long long* marg,
                                        double* y, long long* phase, long long* link, double* scatter,
                                        const char** err);
extern "C" int pspin_deeper_counts(int N, int NT, int nrep, int nsnap, const double* configs, int nbins, int nbins_a2,
                                   double a2_max, const int32_t* quartets, int M, int64_t* marg, double* ipr_terms,
                                   int64_t* phase, int64_t* link, double* scatter) {
    const char* err = nullptr;
    const int rc = pspin_deeper_counts_impl(N, NT, nrep, nsnap, configs, nbins, nbins_a2,
                                            nbins_a2 > 0 ? a2_max / nbins_a2 : 0.0, quartets, M,
                                            reinterpret_cast<long long*>(marg), ipr_terms,
                                            reinterpret_cast<long long*>(phase), reinterpret_cast<long long*>(link),
                                            scatter, &err);
    if (rc == 1) return fail(PSPIN_ERR_ARG, "%s", err);
    if (rc) return fail(PSPIN_ERR_CUDA, "pspin_deeper_counts: %s", err);
    return PSPIN_OK;
}

extern "C" int pspin_multi_overlap_impl(int N, int NT, int nrep, int nsnap, const double* configs,
                                        const int32_t* snaps, int nit, double* out, const char** err);
extern "C" int pspin_multi_overlap(int N, int NT, int nrep, int nsnap, const double* configs, const int32_t* snaps,
                                   int nit, double* out) {
    const char* err = nullptr;
    const int rc = pspin_multi_overlap_impl(N, NT, nrep, nsnap, configs, snaps, nit, out, &err);
    if (rc == 1) return fail(PSPIN_ERR_ARG, "%s", err);
    if (rc) return fail(PSPIN_ERR_CUDA, "pspin_multi_overlap: %s", err);
    return PSPIN_OK;
}

extern "C" int pspin_exchange_host(int n_samples, int NT, int nrep, const double* beta_sched, const double* energy,
                                   const int64_t* rep_off, int32_t* perm, uint64_t* drand_state, int64_t* ex_acc,
                                   int64_t* ex_prop, double* betas) {
    if (n_samples < 0 || NT < 2 || nrep < 1 || !beta_sched || !energy || !rep_off || !perm || !drand_state ||
        !ex_acc || !ex_prop)
        return fail(PSPIN_ERR_ARG, "pspin_exchange_host: bad arguments");
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n_samples; k++) {
        int32_t* pm = perm + (size_t)k * NT * nrep;
        const double* E = energy + rep_off[k];
        uint64_t st = drand_state[k];
        int64_t* acc = ex_acc + (size_t)k * (NT - 1);
        int64_t* prop = ex_prop + (size_t)k * (NT - 1);
        for (int t = 0; t < NT - 1; t++) {
            const double db = beta_sched[t] - beta_sched[t + 1];
            for (int r = 0; r < nrep; r++) {
                const int32_t a = pm[t * nrep + r], b = pm[(t + 1) * nrep + r];
                const double delta = db * (E[a] - E[b]);
                prop[t]++;
                bool ok = delta >= 0.0;
                if (!ok) ok = drand48_next(st) < std::exp(delta);
                if (ok) {
                    acc[t]++;
                    pm[t * nrep + r] = b;
                    pm[(t + 1) * nrep + r] = a;
                }
            }
        }
        drand_state[k] = st;
        if (betas)
            for (int t = 0; t < NT; t++)
                for (int r = 0; r < nrep; r++) betas[rep_off[k] + pm[t * nrep + r]] = beta_sched[t];
    }
    return PSPIN_OK;
}

extern "C" int pspin_pt_shape(pspin_state* s, int* NT, int* nrep_per_temp, int* pt_freq) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (NT) *NT = s->pt_NT;
    if (nrep_per_temp) *nrep_per_temp = s->pt_nrep;
    if (pt_freq) *pt_freq = s->pt_freq;
    return PSPIN_OK;
}

extern "C" int pspin_pt_sweeps_done(pspin_state* s, int64_t* sweeps) {
    if (!s || !sweeps) return fail(PSPIN_ERR_ARG, "null argument");
    *sweeps = s->sweeps_done;
    return PSPIN_OK;
}

// ------------------------------------------------------------------ all-site fields
static int tc_prepare(pspin_state* s, int sample) {
    if (s->tc_sample == sample) return PSPIN_OK;
    const SampleHost& h = s->hs[sample];
    const SampleDev& d = s->sd[sample];
    const int N = h.N, R = h.R;
    const int npairs = N * (N - 1) / 2;
    const int M = (npairs + 127) / 128 * 128, Kp = (npairs + 63) / 64 * 64, NC = (2 * R + 7) / 8 * 8;
    for (void* p : {(void*)s->d_tc_w, (void*)s->d_tc_x, (void*)s->d_tc_f, s->d_tc_ws, (void*)s->d_tc_h,
                    (void*)s->d_f64_h, (void*)s->d_tc_e})
        if (p) cudaFree(p);
    s->d_tc_w = nullptr; s->d_tc_x = nullptr; s->d_tc_f = nullptr; s->d_tc_ws = nullptr;
    s->d_tc_h = nullptr; s->d_f64_h = nullptr; s->d_tc_e = nullptr;
    s->tc_sample = -1;
    // symmetric pair-space couplings Ws[P][Q] = W[P][Q] + W[Q][P] from the FP64 table
    std::vector<Q64> q((size_t)d.nq);
    if (d.nq) CK(cudaMemcpyAsync(q.data(), s->d_q64 + d.q_off, d.nq * sizeof(Q64), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    std::vector<float> ws((size_t)M * Kp, 0.0f);
    static const int U[3][2] = {{0, 1}, {0, 3}, {0, 2}}, C[3][2] = {{2, 3}, {1, 2}, {1, 3}};
    auto pidx = [](int a, int b) { return a < b ? b * (b - 1) / 2 + a : a * (a - 1) / 2 + b; };
    for (const Q64& e : q) {
        const int ch = e.lch >> 14;
        const int v[4] = {e.i, e.j, e.k, e.lch & 0x3FFF};
        const int P = pidx(v[U[ch][0]], v[U[ch][1]]), Q = pidx(v[C[ch][0]], v[C[ch][1]]);
        ws[(size_t)P * Kp + Q] += (float)e.g;
        ws[(size_t)Q * Kp + P] += (float)e.g;
    }
    float* d_ws32 = nullptr;
    TRY(dalloc(&d_ws32, ws.size()));
    int rc = dalloc(&s->d_tc_w, (size_t)M * 3 * Kp);
    if (rc == PSPIN_OK) rc = dalloc(&s->d_tc_x, (size_t)NC * 3 * Kp);
    if (rc == PSPIN_OK) rc = dalloc(&s->d_tc_f, (size_t)M * NC);
    if (rc == PSPIN_OK) rc = dalloc(&s->d_tc_h, (size_t)R * N);
    if (rc == PSPIN_OK) rc = dalloc(&s->d_f64_h, (size_t)R * N);
    if (rc == PSPIN_OK) rc = dalloc(&s->d_tc_e, (size_t)2 * R);
    if (rc == PSPIN_OK) {
        cudaError_t e = cudaMemcpyAsync(d_ws32, ws.data(), ws.size() * sizeof(float), cudaMemcpyHostToDevice, s->st);
        if (e == cudaSuccess) e = launch_split_ws(d_ws32, s->d_tc_w, M, Kp, s->st);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_tc_x, 0, (size_t)NC * 3 * Kp * sizeof(__nv_bfloat16), s->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
        if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "pair-space couplings: %s", cudaGetErrorString(e));
    }
    cudaFree(d_ws32);
    if (rc != PSPIN_OK) return rc;
    size_t need = 0;
    CK(tc_gemm(M, NC, 3 * Kp, nullptr, nullptr, nullptr, nullptr, 0, s->st, &need));
    if (need) TRY(dalloc((char**)&s->d_tc_ws, need));
    s->tc_ws_bytes = need;
    s->tc_sample = sample;
    s->tc_M = M;
    s->tc_Kp = Kp;
    s->tc_NC = NC;
    return PSPIN_OK;
}

// All-site fields and energies of one dense sample on the tensor cores:
// split-BF16 pair operands, the sm100 GEMM, then fields and E2 / E4
// (d_tc_h [R][N], d_tc_e [E2 of R | E4 of R]), enqueued on the stream.
static int tc_fields(pspin_state* s, int sample) {
    const SampleHost& hs = s->hs[sample];
    const SampleDev& d = s->sd[sample];
    const int N = hs.N, R = hs.R;
    const float2* spins = s->d_spins + d.spin_off;
    TRY(tc_prepare(s, sample));
    const int npairs = N * (N - 1) / 2;
    CK(launch_pair_split(spins, N, R, npairs, s->tc_Kp, s->d_tc_x, s->st));
    CK(tc_gemm(s->tc_M, s->tc_NC, 3 * s->tc_Kp, s->d_tc_w, s->d_tc_x, s->d_tc_f, s->d_tc_ws, s->tc_ws_bytes, s->st,
               nullptr));
    CK(launch_site_fields(spins, N, R, s->d_tc_f, s->tc_NC, s->d_g2 + d.g2_off, hs.h2_active, s->d_tc_h, s->d_tc_e,
                          s->d_tc_e + R, s->st));
    s->kernel_launches += 3;
    return PSPIN_OK;
}

// Periodic resync.  FP64 (default): renormalise, full FP64 energies, running
// energy overwritten.  Tensor cores (one dense sample): renormalise in FP64,
// then energies from the split-BF16 contraction.  Both record
// |E_running - E_recomputed| per replica first.
static int do_resync(pspin_state* s) {
    if (s->opt.resync_method != PSPIN_RESYNC_TC) return run_energy(s, nullptr, nullptr, true, true);
    EnergyParams p{};
    p.samples = s->d_samples;
    p.units = s->d_units;
    p.spins = s->d_spins;
    p.quartets = s->d_q64;
    p.g2 = s->d_g2;
    p.target = s->d_target;
    p.renorm_only = 1;
    CK(launch_energy(p, (int)s->units.size(), s->max_N, s->st));
    s->kernel_launches++;
    TRY(tc_fields(s, 0));
    const int R = s->hs[0].R;
    std::vector<double> run(R), e(2 * (size_t)R), drift(R);
    CK(cudaMemcpyAsync(run.data(), s->d_E, R * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(e.data(), s->d_tc_e, 2 * R * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int r = 0; r < R; r++) {
        const double et = e[r] + e[R + r];
        drift[r] = std::fabs(run[r] - et);
        run[r] = et;
    }
    CK(cudaMemcpyAsync(s->d_E, run.data(), R * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_drift, drift.data(), R * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_resync_drift(pspin_state* s, double* drift) {
    if (!s || !drift) return fail(PSPIN_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(drift, s->d_drift, s->R_tot * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_local_fields(pspin_state* s, int sample, int method, double* h, double* energy) {
    if (!s || !h || sample < 0 || sample >= s->S) return fail(PSPIN_ERR_ARG, "bad arguments");
    if (s->variant != PSPIN_DENSE) return fail(PSPIN_ERR_UNSUPPORTED, "all-site fields: dense variant only");
    const SampleHost& hs = s->hs[sample];
    const SampleDev& d = s->sd[sample];
    const int N = hs.N, R = hs.R;
    const float2* spins = s->d_spins + d.spin_off;
    const double* g2 = s->d_g2 + d.g2_off;
    std::vector<double> e(2 * (size_t)R, 0.0);
    if (method == PSPIN_FIELDS_FP64) {
        if (!s->d_f64_h || s->tc_sample != sample) {
            // fields only: the scratch of the tensor-core path is not needed
            if (s->d_f64_h) cudaFree(s->d_f64_h);
            s->d_f64_h = nullptr;
            TRY(dalloc(&s->d_f64_h, (size_t)R * N));
            s->tc_sample = -2;   // the tensor-core buffers (if any) belong to no sample now
        }
        CK(launch_fp64_fields(spins, N, R, s->d_q64 + d.q_off, d.nq, g2, hs.h2_active, s->d_f64_h, s->st));
        s->kernel_launches++;
        std::vector<double2> hv((size_t)R * N);
        CK(cudaMemcpyAsync(hv.data(), s->d_f64_h, hv.size() * sizeof(double2), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        for (size_t t = 0; t < hv.size(); t++) { h[2 * t] = hv[t].x; h[2 * t + 1] = hv[t].y; }
        if (energy) {
            std::vector<double> e2(R), e4(R);
            TRY(run_energy(s, s->d_e2, s->d_e4, false, false));
            CK(cudaMemcpyAsync(e2.data(), s->d_e2 + d.rep_off, R * sizeof(double), cudaMemcpyDeviceToHost, s->st));
            CK(cudaMemcpyAsync(e4.data(), s->d_e4 + d.rep_off, R * sizeof(double), cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            for (int r = 0; r < R; r++) energy[r] = e2[r] + e4[r];
        }
        return PSPIN_OK;
    }
    if (method != PSPIN_FIELDS_TC_BF16X3) return fail(PSPIN_ERR_ARG, "unknown field method %d", method);
    TRY(tc_fields(s, sample));
    std::vector<float2> hv((size_t)R * N);
    CK(cudaMemcpyAsync(hv.data(), s->d_tc_h, hv.size() * sizeof(float2), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(e.data(), s->d_tc_e, 2 * R * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (size_t t = 0; t < hv.size(); t++) { h[2 * t] = hv[t].x; h[2 * t + 1] = hv[t].y; }
    if (energy)
        for (int r = 0; r < R; r++) energy[r] = e[r] + e[R + r];
    return PSPIN_OK;
}

// ------------------------------------------------------------------ learned proposal
// Pair sub-lists for the two-pass sweep: rebuilt from the FP64 quartet table
// (same couplings, rounded to FP32 like the site lists) and appended to the
// entry and chunk arrays; d_pair_chunks indexes them per sample.  The site
// lists of samples without tiles are appended as well in the group format
// (header + entries: the same groups and arithmetic as the records), which
// the two-pass kernel reads faster; d_site_chunks_g indexes them like
// d_site_chunks (tile samples keep their tiles).
static int ensure_pair_lists(pspin_state* s) {
    if (s->d_pair_chunks) return PSPIN_OK;
    const int n = s->S;
    std::vector<std::vector<Q64>> q(n);
    for (int k = 0; k < n; k++) {
        q[k].resize((size_t)s->sd[k].nq);
        if (s->sd[k].nq)
            CK(cudaMemcpyAsync(q[k].data(), s->d_q64 + s->sd[k].q_off, q[k].size() * sizeof(Q64),
                               cudaMemcpyDeviceToHost, s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    std::vector<SiteLists> pl(n), gl(n);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < n; k++) {
        std::vector<QuartetRec> recs(q[k].size());
        for (size_t t = 0; t < q[k].size(); t++) {
            const Q64& e = q[k][t];
            recs[t] = QuartetRec{e.i, e.j, e.k, e.lch & 0x3fff, e.lch >> 14, e.g};
        }
        std::vector<Q64>().swap(q[k]);
        build_pair_lists(s->hs[k].N, s->hs[k].g2re.data(), s->hs[k].h2_active, recs, pl[k]);
        if (!s->hs[k].fc_tiles) build_site_lists(s->hs[k].N, s->hs[k].g2re.data(), s->hs[k].h2_active, recs, gl[k], false);
    }
    int64_t ent_new = 0, chunk_new = 0, idx_total = 0, split_total = 0;
    for (int k = 0; k < n; k++) {
        ent_new += (int64_t)pl[k].entries.size() + (int64_t)gl[k].entries.size();
        chunk_new += (int64_t)pl[k].chunk_start.size() + (int64_t)gl[k].chunk_start.size();
        idx_total += (int64_t)pl[k].site_chunks.size();
        split_total += (int64_t)s->hs[k].N * (kSplit + 1);
    }
    std::vector<int> scg((size_t)split_total);     // group-format site chunk table, tile samples as they are
    if (split_total)
        CK(cudaMemcpyAsync(scg.data(), s->d_site_chunks, scg.size() * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (s->chunk_total + chunk_new >= (1ll << 31)) return fail(PSPIN_ERR_ARG, "too many list chunks for the pair sub-lists");
    std::vector<int2> ent((size_t)ent_new);
    std::vector<int64_t> cs((size_t)chunk_new + 1);
    std::vector<int> pc((size_t)idx_total);
    std::vector<int64_t> pair_off(n);
    int64_t eoff = 0, coff = 0, ioff = 0;
    for (int k = 0; k < n; k++) {
        std::copy(pl[k].entries.begin(), pl[k].entries.end(), ent.begin() + eoff);
        for (size_t t = 0; t < pl[k].chunk_start.size(); t++) cs[coff + t] = pl[k].chunk_start[t] + eoff + s->ent_total;
        for (size_t t = 0; t < pl[k].site_chunks.size(); t++)
            pc[ioff + t] = (int)(pl[k].site_chunks[t] + coff + s->chunk_total);
        pair_off[k] = ioff;
        eoff += (int64_t)pl[k].entries.size();
        coff += (int64_t)pl[k].chunk_start.size();
        ioff += (int64_t)pl[k].site_chunks.size();
        pl[k] = SiteLists();
        if (!gl[k].entries.empty()) {
            std::copy(gl[k].entries.begin(), gl[k].entries.end(), ent.begin() + eoff);
            for (size_t t = 0; t < gl[k].chunk_start.size(); t++) cs[coff + t] = gl[k].chunk_start[t] + eoff + s->ent_total;
            for (size_t t = 0; t < gl[k].site_chunks.size(); t++)
                scg[s->sd[k].split_off + t] = (int)(gl[k].site_chunks[t] + coff + s->chunk_total);
            eoff += (int64_t)gl[k].entries.size();
            coff += (int64_t)gl[k].chunk_start.size();
        }
        gl[k] = SiteLists();
    }
    cs[chunk_new] = s->ent_total + ent_new;
    int2* d_ent = nullptr;
    int64_t* d_cs = nullptr;
    int* d_pc = nullptr;
    int* d_scg = nullptr;
    int rc;
    if ((rc = dalloc(&d_ent, (size_t)(s->ent_total + ent_new))) ||
        (rc = dalloc(&d_cs, (size_t)(s->chunk_total + chunk_new + 1))) || (rc = dalloc(&d_pc, (size_t)idx_total)) ||
        (rc = dalloc(&d_scg, (size_t)std::max<int64_t>(split_total, 1)))) {
        cudaFree(d_ent); cudaFree(d_cs); cudaFree(d_pc); cudaFree(d_scg);
        return rc;
    }
    std::vector<SampleDev> sd = s->sd;
    for (int k = 0; k < n; k++) sd[k].pair_off = pair_off[k];
    cudaError_t e = cudaMemcpyAsync(d_ent, s->d_entries, s->ent_total * sizeof(int2), cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_ent + s->ent_total, ent.data(), ent.size() * sizeof(int2), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_cs, s->d_chunk_start, s->chunk_total * sizeof(int64_t), cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_cs + s->chunk_total, cs.data(), cs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_pc, pc.data(), pc.size() * sizeof(int), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess && split_total)
        e = cudaMemcpyAsync(d_scg, scg.data(), scg.size() * sizeof(int), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->d_samples, sd.data(), sd.size() * sizeof(SampleDev), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) {
        cudaFree(d_ent); cudaFree(d_cs); cudaFree(d_pc); cudaFree(d_scg);
        return fail(PSPIN_ERR_CUDA, "pair sub-list upload: %s", cudaGetErrorString(e));
    }
    s->sd = sd;
    cudaFree(s->d_entries);
    cudaFree(s->d_chunk_start);
    s->d_entries = d_ent;
    s->d_chunk_start = d_cs;
    s->d_pair_chunks = d_pc;
    s->d_site_chunks_g = d_scg;
    s->ent_total += ent_new;
    s->chunk_total += chunk_new;
    return PSPIN_OK;
}

extern "C" int pspin_set_proposal(pspin_state* s, int proposal) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (proposal < PSPIN_PROPOSAL_PLAIN || proposal > PSPIN_PROPOSAL_LEARNED)
        return fail(PSPIN_ERR_ARG, "unknown proposal %d", proposal);
    if (proposal != PSPIN_PROPOSAL_PLAIN && s->variant != PSPIN_DENSE)
        return fail(PSPIN_ERR_UNSUPPORTED, "the learned proposal is built for the dense (spherical) variant");
    if (proposal == PSPIN_PROPOSAL_LEARNED && !s->d_wbf)
        return fail(PSPIN_ERR_STATE, "pspin_learn_init has not been called");
    if (proposal != PSPIN_PROPOSAL_PLAIN) TRY(ensure_pair_lists(s));
    if (proposal != s->proposal) drop_graph(s);
    s->proposal = proposal;
    return PSPIN_OK;
}

extern "C" int pspin_learn_init(pspin_state* s, uint64_t seed, int capacity, float record_prob) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (capacity < 1) return fail(PSPIN_ERR_ARG, "record capacity must be >= 1");
    drop_graph(s);
    for (void* p : {(void*)s->d_w32, (void*)s->d_adam_m, (void*)s->d_adam_v, (void*)s->d_grad, (void*)s->d_wbf,
                    (void*)s->d_records, (void*)s->d_rec_count})
        if (p) cudaFree(p);
    s->d_w32 = s->d_adam_m = s->d_adam_v = s->d_grad = nullptr;
    s->d_wbf = nullptr;
    s->d_records = nullptr;
    s->d_rec_count = nullptr;
    const int P = kMlpParamsHost;
    int rc;
    if ((rc = dalloc(&s->d_w32, P)) || (rc = dalloc(&s->d_adam_m, P)) || (rc = dalloc(&s->d_adam_v, P)) ||
        (rc = dalloc(&s->d_grad, P)) || (rc = dalloc(&s->d_wbf, P)) ||
        (rc = dalloc(&s->d_records, (size_t)capacity * kRecordFloatsHost)) || (rc = dalloc(&s->d_rec_count, 1)))
        return rc;
    // Xavier-uniform weights; biases 0 except the mixtures: means spread over
    // the circle, concentrations low (kappa ~ 1)
    std::vector<float> w(P, 0.0f);
    uint64_t st = seed;
    auto uni = [&]() { return (double)(splitmix64(st) >> 11) / 9007199254740992.0; };
    auto fill = [&](int off, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int t = 0; t < fan_out * fan_in; t++) w[off + t] = (float)((2.0 * uni() - 1.0) * a);
    };
    fill(0, 64, 8);
    fill(8 * 64 + 64, 64, 64);
    const int offW3 = 8 * 64 + 64 + 64 * 64 + 64, offB3 = offW3 + 26 * 64;
    fill(offW3, 26, 64);
    for (int t = 0; t < 26 * 64; t++) w[offW3 + t] *= 0.1f;
    for (int sdx = 0; sdx < 2; sdx++)
        for (int k = 0; k < 4; k++) {
            w[offB3 + 2 + 12 * sdx + 4 + k] = (float)(k * 1.5707963267948966 - 2.356194490192345);
            w[offB3 + 2 + 12 * sdx + 8 + k] = -3.9f;
        }
    CK(cudaMemcpyAsync(s->d_w32, w.data(), P * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->d_adam_m, 0, P * sizeof(float), s->st));
    CK(cudaMemsetAsync(s->d_adam_v, 0, P * sizeof(float), s->st));
    CK(cudaMemsetAsync(s->d_rec_count, 0, sizeof(unsigned long long), s->st));
    CK(launch_to_bf16(s->d_w32, s->d_wbf, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->rec_cap = capacity;
    s->rec_prob = record_prob;
    s->adam_t = 0;
    s->learn_seed = seed;
    return PSPIN_OK;
}

extern "C" int pspin_learn_params(pspin_state* s, float* get, const float* set) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (!s->d_w32) return fail(PSPIN_ERR_STATE, "pspin_learn_init has not been called");
    if (get) CK(cudaMemcpyAsync(get, s->d_w32, kMlpParamsHost * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    if (set) {
        CK(cudaMemcpyAsync(s->d_w32, set, kMlpParamsHost * sizeof(float), cudaMemcpyHostToDevice, s->st));
        CK(launch_to_bf16(s->d_w32, s->d_wbf, s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

static int ensure_save(pspin_state* s, int n) {
    if (n <= s->save_cap) return PSPIN_OK;
    cudaFree(s->d_save);
    cudaFree(s->d_loss);
    cudaFree(s->d_idx);
    s->d_save = nullptr; s->d_loss = nullptr; s->d_idx = nullptr;
    s->save_cap = 0;
    int rc;
    if ((rc = dalloc(&s->d_save, (size_t)n * kSaveFloatsHost)) || (rc = dalloc(&s->d_loss, n)) ||
        (rc = dalloc(&s->d_idx, n)))
        return rc;
    s->save_cap = n;
    return PSPIN_OK;
}

extern "C" int pspin_learn_train(pspin_state* s, int steps, int batch, float lr, double* mean_loss) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (!s->d_w32) return fail(PSPIN_ERR_STATE, "pspin_learn_init has not been called");
    if (steps < 0 || batch < 1) return fail(PSPIN_ERR_ARG, "bad steps/batch");
    unsigned long long cnt = 0;
    CK(cudaMemcpyAsync(&cnt, s->d_rec_count, sizeof(cnt), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const unsigned long long filled = cnt < (unsigned long long)s->rec_cap ? cnt : (unsigned long long)s->rec_cap;
    if (filled == 0) return fail(PSPIN_ERR_STATE, "no training records yet");
    TRY(ensure_save(s, batch));
    for (int it = 0; it < steps; it++) {
        CK(launch_sample_index(s->d_idx, batch, filled, s->learn_seed ^ 0x5eedULL, (uint32_t)s->adam_t, s->st));
        CK(launch_mlp_fwd_bwd(s->d_w32, s->d_records, s->d_idx, batch, s->d_save, s->d_loss, s->st));
        CK(launch_mlp_grad(s->d_save, batch, s->d_grad, s->st));
        s->adam_t++;
        CK(launch_adam(s->d_w32, s->d_adam_m, s->d_adam_v, s->d_grad, s->d_wbf, lr, s->adam_t, s->st));
        s->kernel_launches += 4;
    }
    if (mean_loss) {
        std::vector<float> l(batch);
        CK(cudaMemcpyAsync(l.data(), s->d_loss, batch * sizeof(float), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        double m = 0.0;
        for (float v : l) m += v;
        *mean_loss = m / batch;
    }
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_learn_records(pspin_state* s, int64_t* n_recorded, float* out, int max) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    if (!s->d_rec_count) return fail(PSPIN_ERR_STATE, "pspin_learn_init has not been called");
    unsigned long long cnt = 0;
    CK(cudaMemcpyAsync(&cnt, s->d_rec_count, sizeof(cnt), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (n_recorded) *n_recorded = (int64_t)cnt;
    if (out && max > 0) {
        const unsigned long long n = std::min<unsigned long long>(
            std::min<unsigned long long>(cnt, (unsigned long long)s->rec_cap), (unsigned long long)max);
        CK(cudaMemcpyAsync(out, s->d_records, n * kRecordFloatsHost * sizeof(float), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    return PSPIN_OK;
}

extern "C" int pspin_learn_loss_grad(pspin_state* s, const float* records, int n, double* loss, float* grad) {
    if (!s || !records || n < 1) return fail(PSPIN_ERR_ARG, "bad arguments");
    if (!s->d_w32) return fail(PSPIN_ERR_STATE, "pspin_learn_init has not been called");
    TRY(ensure_save(s, n));
    float* d_rec = nullptr;
    TRY(dalloc(&d_rec, (size_t)n * kRecordFloatsHost));
    cudaError_t e = cudaMemcpyAsync(d_rec, records, (size_t)n * kRecordFloatsHost * sizeof(float),
                                    cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = launch_mlp_fwd_bwd(s->d_w32, d_rec, nullptr, n, s->d_save, s->d_loss, s->st);
    if (e == cudaSuccess) e = launch_mlp_grad(s->d_save, n, s->d_grad, s->st);
    std::vector<float> l(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.data(), s->d_loss, n * sizeof(float), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess && grad)
        e = cudaMemcpyAsync(grad, s->d_grad, kMlpParamsHost * sizeof(float), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(d_rec);
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "loss/grad: %s", cudaGetErrorString(e));
    if (loss) {
        double m = 0.0;
        for (float v : l) m += v;
        *loss = m / n;
    }
    return PSPIN_OK;
}

// ------------------------------------------------------------------ checkpoint / resume
// A binary file with everything that continues a chain bit for bit: FP32
// amplitudes, running energies, counters, betas, the device sweep index
// (which keys the pair and move streams), the resync phase, the PT state and
// the learned network with its Adam moments.  Loading checks that the handle
// was built from the same configurations (variant, N, replicas, seed, FMC).
static const char kCkMagic[8] = {'P', 'S', 'P', 'I', 'N', 'C', 'K', '2'};

namespace {
struct CkFile {
    FILE* f = nullptr;
    bool ok = true;
    ~CkFile() { if (f) fclose(f); }
    void put(const void* p, size_t n) { if (ok && n && fwrite(p, 1, n, f) != n) ok = false; }
    void get(void* p, size_t n) { if (ok && n && fread(p, 1, n, f) != n) ok = false; }
    template <class T> void put(const T& v) { put(&v, sizeof(T)); }
    template <class T> void get(T& v) { get(&v, sizeof(T)); }
};
}  // namespace

template <class T>
static int dev_to_file(pspin_state* s, CkFile& f, const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) CK(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    f.put(h.data(), n * sizeof(T));
    return PSPIN_OK;
}

template <class T>
static int file_to_dev(pspin_state* s, CkFile& f, T* d, size_t n) {
    std::vector<T> h(n);
    f.get(h.data(), n * sizeof(T));
    if (!f.ok) return fail(PSPIN_ERR_ARG, "checkpoint file is truncated");
    if (n) CK(cudaMemcpyAsync(d, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return PSPIN_OK;
}

extern "C" int pspin_checkpoint_save(pspin_state* s, const char* path) {
    if (!s || !path) return fail(PSPIN_ERR_ARG, "null argument");
    CkFile f;
    f.f = fopen(path, "wb");
    if (!f.f) return fail(PSPIN_ERR_ARG, "cannot open %s for writing", path);
    CK(cudaStreamSynchronize(s->st));
    long long counter = 0;
    CK(cudaMemcpy(&counter, s->d_sweep_counter, sizeof(counter), cudaMemcpyDeviceToHost));
    f.put(kCkMagic, sizeof(kCkMagic));
    f.put((int32_t)s->variant);
    f.put((int32_t)s->opt.disorder_stream);   // which couplings the chain ran on
    f.put((int32_t)s->S);
    f.put((int64_t)s->R_tot);
    f.put((int64_t)s->spin_total);
    for (const SampleHost& h : s->hs) {
        f.put((int32_t)h.N);
        f.put((int32_t)h.R);
        f.put((uint64_t)h.cfg.seed);
        f.put((int32_t)h.cfg.fmc_mode);
    }
    f.put((int64_t)s->sweeps_done);
    f.put((int64_t)s->since_resync);
    f.put((int64_t)counter);
    f.put((int32_t)s->proposal);
    f.put((int32_t)s->warps);          // block shapes: they fix the summation order
    f.put((int32_t)s->cluster);
    f.put((int32_t)s->warps2);
    f.put((int32_t)s->cluster2);
    TRY(dev_to_file(s, f, s->d_spins, (size_t)s->spin_total));
    TRY(dev_to_file(s, f, s->d_E, (size_t)s->R_tot));
    TRY(dev_to_file(s, f, s->d_beta, (size_t)s->R_tot));
    TRY(dev_to_file(s, f, s->d_target, (size_t)s->R_tot));
    TRY(dev_to_file(s, f, s->d_acc, (size_t)s->R_tot));
    TRY(dev_to_file(s, f, s->d_prop, (size_t)s->R_tot));
    f.put((int32_t)s->pt_NT);
    f.put((int32_t)s->pt_nrep);
    f.put((int32_t)s->pt_freq);
    if (s->pt_NT >= 2) {
        const size_t NT = s->pt_NT, nr = s->pt_nrep, S = s->S;
        TRY(dev_to_file(s, f, s->d_beta_sched, NT));
        TRY(dev_to_file(s, f, s->d_perm, S * NT * nr));
        TRY(dev_to_file(s, f, s->d_drand, S));
        TRY(dev_to_file(s, f, s->d_ex_acc, S * (NT - 1)));
        TRY(dev_to_file(s, f, s->d_ex_prop, S * (NT - 1)));
    }
    const int32_t has_net = s->d_w32 ? 1 : 0;
    f.put(has_net);
    if (has_net) {
        f.put((int32_t)s->adam_t);
        f.put((uint64_t)s->learn_seed);
        f.put((float)s->rec_prob);
        f.put((int32_t)s->rec_cap);
        TRY(dev_to_file(s, f, s->d_w32, (size_t)kMlpParamsHost));
        TRY(dev_to_file(s, f, s->d_adam_m, (size_t)kMlpParamsHost));
        TRY(dev_to_file(s, f, s->d_adam_v, (size_t)kMlpParamsHost));
    }
    if (!f.ok) return fail(PSPIN_ERR_ARG, "write to %s failed", path);
    return PSPIN_OK;
}

// Reads and checks the whole file into host buffers before it changes
// anything, so a rejected or truncated file leaves the handle as it was.
extern "C" int pspin_checkpoint_load(pspin_state* s, const char* path) {
    if (!s || !path) return fail(PSPIN_ERR_ARG, "null argument");
    CkFile f;
    f.f = fopen(path, "rb");
    if (!f.f) return fail(PSPIN_ERR_ARG, "cannot open %s", path);
    char magic[8];
    f.get(magic, sizeof(magic));
    if (!f.ok || std::memcmp(magic, kCkMagic, sizeof(magic)) != 0) return fail(PSPIN_ERR_ARG, "%s is not a checkpoint", path);
    int32_t variant = 0, dstream = 0, S = 0;
    int64_t R_tot = 0, spin_total = 0;
    f.get(variant); f.get(dstream); f.get(S); f.get(R_tot); f.get(spin_total);
    if (!f.ok || variant != s->variant || S != s->S || R_tot != s->R_tot || spin_total != s->spin_total ||
        dstream != s->opt.disorder_stream)
        return fail(PSPIN_ERR_ARG,
                    "checkpoint does not match this handle (variant, coupling source, samples or replicas)");
    for (const SampleHost& h : s->hs) {
        int32_t N = 0, R = 0, fmc = 0;
        uint64_t seed = 0;
        f.get(N); f.get(R); f.get(seed); f.get(fmc);
        if (!f.ok || N != h.N || R != h.R || seed != (uint64_t)h.cfg.seed || fmc != h.cfg.fmc_mode)
            return fail(PSPIN_ERR_ARG, "checkpoint does not match this handle (a sample's N, replicas, seed or FMC)");
    }
    int64_t sweeps_done = 0, since_resync = 0, counter = 0;
    int32_t proposal = 0, warps = 0, cluster = 0, warps2 = 0, cluster2 = 0;
    f.get(sweeps_done); f.get(since_resync); f.get(counter); f.get(proposal);
    f.get(warps); f.get(cluster); f.get(warps2); f.get(cluster2);
    if (!f.ok || warps < 1 || warps > 8 || warps2 < 1 || warps2 > 8 || cluster < 0 || cluster > 16 || cluster2 < 1 ||
        cluster2 > 16 || proposal < PSPIN_PROPOSAL_PLAIN || proposal > PSPIN_PROPOSAL_LEARNED)
        return fail(PSPIN_ERR_ARG, "checkpoint file is truncated or corrupt");
    const size_t R = (size_t)s->R_tot;
    std::vector<float2> spins((size_t)s->spin_total);
    std::vector<double> E(R), betas(R), target(R);
    std::vector<long long> acc(R), prop(R);
    f.get(spins.data(), spins.size() * sizeof(float2));
    f.get(E.data(), R * sizeof(double));
    f.get(betas.data(), R * sizeof(double));
    f.get(target.data(), R * sizeof(double));
    f.get(acc.data(), R * sizeof(long long));
    f.get(prop.data(), R * sizeof(long long));
    int32_t NT = 0, nrep = 0, freq = 0;
    f.get(NT); f.get(nrep); f.get(freq);
    if (!f.ok) return fail(PSPIN_ERR_ARG, "checkpoint file is truncated");
    if (NT == 1 || NT < 0 || (NT >= 2 && (nrep < 1 || freq < 1)))
        return fail(PSPIN_ERR_ARG, "checkpoint file is corrupt (PT shape NT=%d nrep=%d pt_freq=%d)", NT, nrep, freq);
    if (NT >= 2)
        for (const SampleHost& h : s->hs)
            if (h.R != NT * nrep) return fail(PSPIN_ERR_ARG, "checkpoint PT shape does not match the samples' replicas");
    const size_t SS = s->S, nt = NT >= 2 ? (size_t)NT : 0, nr = NT >= 2 ? (size_t)nrep : 0;
    std::vector<double> sched(nt);
    std::vector<int> perm(SS * nt * nr);
    std::vector<unsigned long long> drand(nt ? SS : 0);
    std::vector<long long> ex_acc(nt ? SS * (nt - 1) : 0), ex_prop(ex_acc.size());
    f.get(sched.data(), sched.size() * sizeof(double));
    f.get(perm.data(), perm.size() * sizeof(int));
    f.get(drand.data(), drand.size() * sizeof(unsigned long long));
    f.get(ex_acc.data(), ex_acc.size() * sizeof(long long));
    f.get(ex_prop.data(), ex_prop.size() * sizeof(long long));
    int32_t has_net = 0, adam_t = 0, cap = 0;
    uint64_t lseed = 0;
    float prob = 0.f;
    f.get(has_net);
    std::vector<float> w32, am, av;
    if (f.ok && has_net) {
        f.get(adam_t); f.get(lseed); f.get(prob); f.get(cap);
        w32.resize(kMlpParamsHost);
        am.resize(kMlpParamsHost);
        av.resize(kMlpParamsHost);
        f.get(w32.data(), w32.size() * sizeof(float));
        f.get(am.data(), am.size() * sizeof(float));
        f.get(av.data(), av.size() * sizeof(float));
    }
    if (!f.ok) return fail(PSPIN_ERR_ARG, "checkpoint file is truncated");
    if (fgetc(f.f) != EOF) return fail(PSPIN_ERR_ARG, "checkpoint file has trailing bytes (corrupt)");
    for (size_t i = 0; i < perm.size(); i++)
        if (perm[i] < 0 || perm[i] >= NT * nrep) return fail(PSPIN_ERR_ARG, "checkpoint file is corrupt (perm)");
    if (proposal == PSPIN_PROPOSAL_LEARNED && !has_net && !s->d_w32)
        return fail(PSPIN_ERR_ARG, "checkpoint uses the learned proposal but holds no network");

    // ---- everything checked: apply
    drop_graph(s);
    CK(cudaMemcpyAsync(s->d_spins, spins.data(), spins.size() * sizeof(float2), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_E, E.data(), R * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_target, target.data(), R * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_acc, acc.data(), R * sizeof(long long), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->d_prop, prop.data(), R * sizeof(long long), cudaMemcpyHostToDevice, s->st));
    if (NT >= 2) {
        TRY(pspin_pt_init(s, NT, nrep, sched.data(), freq));
        CK(cudaMemcpyAsync(s->d_perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->d_drand, drand.data(), drand.size() * sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->d_ex_acc, ex_acc.data(), ex_acc.size() * sizeof(long long), cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->d_ex_prop, ex_prop.data(), ex_prop.size() * sizeof(long long), cudaMemcpyHostToDevice,
                           s->st));
    } else if (s->pt_NT >= 2) {
        // the saved chain ran without PT: the handle's PT state would resume with a wrong perm
        CK(cudaStreamSynchronize(s->st));
        cudaFree(s->d_beta_sched); cudaFree(s->d_perm); cudaFree(s->d_drand); cudaFree(s->d_ex_acc); cudaFree(s->d_ex_prop);
        s->d_beta_sched = nullptr; s->d_perm = nullptr; s->d_drand = nullptr; s->d_ex_acc = nullptr; s->d_ex_prop = nullptr;
        s->pt_NT = s->pt_nrep = s->pt_freq = 0;
        s->obs_cap = 0;
    }
    CK(cudaMemcpyAsync(s->d_beta, betas.data(), R * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (has_net) {
        TRY(pspin_learn_init(s, lseed, std::max(cap, 1), prob));
        CK(cudaMemcpyAsync(s->d_w32, w32.data(), w32.size() * sizeof(float), cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->d_adam_m, am.data(), am.size() * sizeof(float), cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->d_adam_v, av.data(), av.size() * sizeof(float), cudaMemcpyHostToDevice, s->st));
        CK(launch_to_bf16(s->d_w32, s->d_wbf, s->st));
        s->adam_t = adam_t;
    }
    TRY(pspin_set_proposal(s, proposal));
    CK(cudaMemcpyAsync(s->d_sweep_counter, &counter, sizeof(counter), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->sweeps_done = sweeps_done;
    s->since_resync = since_resync;
    s->warps = warps;
    s->cluster = cluster;
    s->warps2 = warps2;
    s->cluster2 = cluster2;
    drop_graph(s);
    return PSPIN_OK;
}

extern "C" int pspin_trace_get(pspin_state* s, pspin_move_record* out, int max_records, int* n_records) {
    if (!s || !out || !n_records) return fail(PSPIN_ERR_ARG, "null argument");
    if (!s->d_trace) return fail(PSPIN_ERR_STATE, "tracing was not enabled at creation");
    const int sample = s->opt.trace_sample;
    const int steps = s->hs[sample].N / 2;
    long long n = (s->sweeps_done - s->trace_sweep0) * steps;
    if (n > s->opt.trace_capacity) n = s->opt.trace_capacity;
    if (n > max_records) n = max_records;
    CK(cudaMemcpyAsync(out, s->d_trace, (size_t)n * sizeof(pspin_move_record), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    *n_records = (int)n;
    return PSPIN_OK;
}

// ------------------------------------------------------------------ stand-alone kernels
extern "C" int pspin_fmc_mask(int N, const double* omega, double gamma, uint8_t* mask_out, int64_t* n_active) {
    if (N < 4 || !omega) return fail(PSPIN_ERR_ARG, "bad arguments");
    const int64_t nq = C4(N);
    double* d_w = nullptr;
    uint8_t* d_m = nullptr;
    unsigned long long* d_c = nullptr;
    int rc;
    if ((rc = dalloc(&d_w, N)) || (rc = dalloc(&d_m, (size_t)nq)) || (rc = dalloc(&d_c, 1))) {
        cudaFree(d_w); cudaFree(d_m); cudaFree(d_c);
        return rc;
    }
    unsigned long long cnt = 0;
    cudaError_t e = cudaMemcpy(d_w, omega, N * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = dev_fmc_mask(d_m, d_w, N, gamma, 0);
    if (e == cudaSuccess) e = dev_popcount(d_m, nq, d_c, 0);
    if (e == cudaSuccess && mask_out) e = cudaMemcpy(mask_out, d_m, (size_t)nq, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&cnt, d_c, sizeof(cnt), cudaMemcpyDeviceToHost);
    cudaFree(d_w); cudaFree(d_m); cudaFree(d_c);
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "fmc mask: %s", cudaGetErrorString(e));
    if (n_active) *n_active = (int64_t)cnt;
    return PSPIN_OK;
}

// ------------------------------------------------------------------ multi-GPU sharding
// Longest-processing-time bin packing of independent samples over shards
// (GPUs): costs N^4 R (one sweep's field work: N/2 moves over site lists of
// ~N^3 terms, for R replicas), taken largest first (ties by index) and each
// given to the least-loaded shard (ties by shard index).  Deterministic, so
// every rank computes the same assignment without communicating.
extern "C" int pspin_shard_samples(int n_samples, const int* N, const int* R, int nshards, int* shard_of) {
    if (n_samples < 0 || nshards < 1 || (n_samples > 0 && (!N || !R || !shard_of)))
        return fail(PSPIN_ERR_ARG, "pspin_shard_samples: bad arguments");
    std::vector<int> order(n_samples);
    std::vector<double> cost(n_samples);
    for (int k = 0; k < n_samples; k++) {
        if (N[k] < 1 || R[k] < 1) return fail(PSPIN_ERR_ARG, "pspin_shard_samples: N and R must be >= 1");
        const double n = (double)N[k];
        cost[k] = n * n * n * n * (double)R[k];
        order[k] = k;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> load(nshards, 0.0);
    for (int k : order) {
        int best = 0;
        for (int r = 1; r < nshards; r++)
            if (load[r] < load[best]) best = r;
        shard_of[k] = best;
        load[best] += cost[k];
    }
    return PSPIN_OK;
}

// ------------------------------------------------------------------ smoothed cube
// smoothed_cube.cu:330-352: nsamples configurations of N amplitudes from one
// cuRAND Philox call of 2 N nsamples normals (seed), each scaled onto
// sum |a|^4 = N on the device; out [nsamples][N][2].
extern "C" int pspin_cube_samples(int N, int nsamples, uint64_t seed, double* out) {
    if (N < 2 || nsamples < 1 || !out) return fail(PSPIN_ERR_ARG, "need N >= 2, nsamples >= 1 and an output");
    const size_t n = 2 * (size_t)N * nsamples;
    double* d = nullptr;
    TRY(dalloc(&d, n));
    int rc = curand_normals(seed, n, d, 0);
    cudaError_t e = cudaSuccess;
    if (rc == PSPIN_OK) e = launch_cube_normalize_many(d, N, nsamples, 0);
    if (rc == PSPIN_OK && e == cudaSuccess) e = cudaMemcpy(out, d, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (rc != PSPIN_OK) return rc;
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "cube samples: %s", cudaGetErrorString(e));
    return PSPIN_OK;
}

// The free walk of smoothed_cube.cu:74-119 on the engine's cube move: the
// start is the reference's init_spins_cube(seed + 9999) (spins_sparse.cu:
// 63-80: cuRAND normals, the shared-memory tree normalisation), rounded to
// FP32; `sweeps` sweeps of N/2 always-accepted moves from the engine's
// streams keyed by seed + 12345; traj [max_saved][N][2] gets the state
// before the walk and after every save_freq-th sweep, *n_saved the count.
extern "C" int pspin_cube_walk(int N, int sweeps, int save_freq, uint64_t seed, double* traj, int max_saved,
                               int* n_saved) {
    if (N < 2 || sweeps < 0 || save_freq < 1 || max_saved < 1 || !traj || !n_saved)
        return fail(PSPIN_ERR_ARG, "need N >= 2, sweeps >= 0, save_freq >= 1 and an output");
    double* d_nrm = nullptr;
    TRY(dalloc(&d_nrm, 2 * (size_t)N));
    std::vector<double> a0(2 * (size_t)N);
    int rc = curand_normals(seed + 9999, 2 * (size_t)N, d_nrm, 0);
    cudaError_t e = cudaSuccess;
    if (rc == PSPIN_OK) e = cudaMemcpy(a0.data(), d_nrm, a0.size() * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_nrm);
    if (rc != PSPIN_OK) return rc;
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "cube walk: %s", cudaGetErrorString(e));
    normalize_host(a0.data(), N, 1, 0);
    std::vector<float2> af(N);
    for (int k = 0; k < N; k++) af[k] = make_float2((float)a0[2 * k], (float)a0[2 * k + 1]);
    uint64_t st = seed + 12345;
    const uint64_t move_key = splitmix64(st), pair_key = splitmix64(st);
    float2* d_a = nullptr;
    double* d_t = nullptr;
    int* d_n = nullptr;
    rc = dalloc(&d_a, N);
    if (rc == PSPIN_OK) rc = dalloc(&d_t, 2 * (size_t)N * max_saved);
    if (rc == PSPIN_OK) rc = dalloc(&d_n, 1);
    if (rc == PSPIN_OK) {
        e = cudaMemcpy(d_a, af.data(), N * sizeof(float2), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = launch_cube_walk(d_a, N, sweeps, save_freq, move_key, pair_key, d_t, max_saved, d_n, 0);
        if (e == cudaSuccess) e = cudaMemcpy(n_saved, d_n, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(traj, d_t, 2 * (size_t)N * std::min(*n_saved, max_saved) * sizeof(double),
                           cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(PSPIN_ERR_CUDA, "cube walk: %s", cudaGetErrorString(e));
    }
    cudaFree(d_a);
    cudaFree(d_t);
    cudaFree(d_n);
    return rc;
}

extern "C" int pspin_quartet_roundtrip(int N, int64_t* n_fail) {
    if (N < 4 || !n_fail) return fail(PSPIN_ERR_ARG, "bad arguments");
    unsigned long long* d = nullptr;
    TRY(dalloc(&d, 1));
    unsigned long long h = 0;
    cudaError_t e = dev_roundtrip(N, C4(N), d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "roundtrip: %s", cudaGetErrorString(e));
    *n_fail = (int64_t)h;
    return PSPIN_OK;
}

// ------------------------------------------------------------------ measurement
extern "C" void* pspin_stream(pspin_state* s) { return s ? (void*)s->st : nullptr; }

extern "C" int pspin_set_profiling(pspin_state* s, int on) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    s->profiling = on != 0;
    s->ev_used = 0;
    s->sweep_launches = 0;
    s->kernel_launches = 0;
    return PSPIN_OK;
}

extern "C" int pspin_get_profile(pspin_state* s, double* ms, int64_t* sweep_launches, int64_t* kernel_launches) {
    if (!s) return fail(PSPIN_ERR_ARG, "null handle");
    CK(cudaStreamSynchronize(s->st));
    double tot = 0.0;
    for (size_t i = 0; i < s->ev_used; i++) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, s->ev_pool[i].first, s->ev_pool[i].second));
        tot += t;
    }
    if (ms) *ms = tot;
    if (sweep_launches) *sweep_launches = s->sweep_launches;
    if (kernel_launches) *kernel_launches = s->kernel_launches;
    s->ev_used = 0;
    s->sweep_launches = 0;
    s->kernel_launches = 0;
    return PSPIN_OK;
}

namespace pspin {
cudaError_t launch_fma_probe(float* out, int blocks, int iters, cudaStream_t st, int paired);
}  // namespace pspin

// FP32 FMA throughput of this GPU: the faster of a scalar (fma.rn.f32) and a
// paired (fma.rn.f32x2) FMA loop, 8 independent chains per thread, 8 CTAs of
// 256 threads per SM, best of 5 timed launches.
extern "C" int pspin_fp32_peak(double* tflops) {
    if (!tflops) return fail(PSPIN_ERR_ARG, "null argument");
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* d = nullptr;
    TRY(dalloc(&d, (size_t)sms * 8 * 1024));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int iters = 1 << 14;
    const int blocks = sms * 8;
    cudaError_t e = cudaSuccess;
    double best_tf = 0.0;
    for (int paired = 0; paired < 2 && e == cudaSuccess; paired++) {
        e = launch_fma_probe(d, blocks, iters, 0, paired);   // warm-up
        float best = 1e30f;
        for (int rep = 0; rep < 5 && e == cudaSuccess; rep++) {
            cudaEventRecord(a, 0);
            e = launch_fma_probe(d, blocks, iters, 0, paired);
            cudaEventRecord(b, 0);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            float t = 0.f;
            cudaEventElapsedTime(&t, a, b);
            if (t > 0.f && t < best) best = t;
        }
        // 256 threads x 8 chains (x 2 lanes when paired) x 2 flop per FMA x iters
        const double flops = (double)blocks * 256 * 8 * (paired ? 2 : 1) * 2.0 * iters;
        if (e == cudaSuccess) best_tf = std::max(best_tf, flops / (best * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return fail(PSPIN_ERR_CUDA, "fma probe: %s", cudaGetErrorString(e));
    *tflops = best_tf;
    return PSPIN_OK;
}

extern "C" const char* pspin_last_error(void) { return g_err.c_str(); }
extern "C" const char* pspin_version(void) { return "pspin-b200 0.1 (sm_100a)"; }
