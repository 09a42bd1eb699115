// ref_bench.cu -- times the reference's own sweep (mc_sweep_pt /
// mc_sparse_sweep_pt) on the GPU, the way its bench_pt_scaling.cu:73-165
// does: a cudaEvent pair around nsweeps calls, each call including its own
// launch and cudaDeviceSynchronize.  Optionally adds the host exchange of
// parallel_tempering.cu:316-352 (3 D2H copies, drand48 loop, 1 H2D) after
// every sweep, i.e. the reference's PT loop without file output.
//
// usage: ref_bench dense|sparse -N n -NT nt -nrepT r [-sweeps s] [-warmup w]
//        [-seed s] [-fmc f] [-gamma g] [-Tmin a] [-Tmax b] [-exchange 0|1]
// prints one line: N NT nrepT sweeps ms_total ms_per_sweep pair_moves_per_s
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "config.h"
#include "mc.h"
#include "mc_sparse.h"

int main(int argc, char** argv) {
    bool sparse = argc > 1 && !strcmp(argv[1], "sparse");
    int N = 32, NT = 20, nr = 4, sweeps = 64, warmup = 4, fmc = 0, ex = 1;
    unsigned long long seed = 42;
    double gamma = 0.0, Tmin = 0.2, Tmax = 1.6;
    for (int i = 2; i < argc; i++) {
        const char* a = argv[i];
        if (i + 1 >= argc) break;
        if (!strcmp(a, "-N")) N = atoi(argv[++i]);
        else if (!strcmp(a, "-NT")) NT = atoi(argv[++i]);
        else if (!strcmp(a, "-nrepT")) nr = atoi(argv[++i]);
        else if (!strcmp(a, "-sweeps")) sweeps = atoi(argv[++i]);
        else if (!strcmp(a, "-warmup")) warmup = atoi(argv[++i]);
        else if (!strcmp(a, "-seed")) seed = strtoull(argv[++i], nullptr, 10);
        else if (!strcmp(a, "-fmc")) fmc = atoi(argv[++i]);
        else if (!strcmp(a, "-gamma")) gamma = atof(argv[++i]);
        else if (!strcmp(a, "-Tmin")) Tmin = atof(argv[++i]);
        else if (!strcmp(a, "-Tmax")) Tmax = atof(argv[++i]);
        else if (!strcmp(a, "-exchange")) ex = atoi(argv[++i]);
    }
    SimConfig cfg = default_config();
    cfg.N = N;
    cfg.nrep = NT * nr;
    cfg.seed = seed;
    cfg.fmc_mode = fmc;
    cfg.gamma = gamma;
    if (fmc > 0 && gamma <= 0.0) cfg.gamma = (fmc == 1) ? 0.0 : 1.0 / (2.0 * (N - 1));
    const int R = NT * nr;
    std::vector<double> bs(NT), betas(R), E(R);
    std::vector<long long> a(R), p(R);
    std::vector<int> perm(R);
    double A = pow(Tmin / Tmax, 1.0 / (NT - 1));
    for (int t = 0; t < NT; t++) bs[t] = 1.0 / (Tmax * pow(A, t));
    for (int t = 0; t < NT; t++)
        for (int r = 0; r < nr; r++) betas[t * nr + r] = bs[t];
    for (int i = 0; i < R; i++) perm[i] = i;
    srand48((long)seed + 5000);
    MCState d{};
    MCStateSparse s{};
    if (sparse) { s = mc_sparse_init(cfg); mc_sparse_set_betas(s, betas.data()); }
    else { d = mc_init(cfg); mc_set_betas(d, betas.data()); }
    auto step = [&]() {
        if (sparse) mc_sparse_sweep_pt(s); else mc_sweep_pt(d);
        if (!ex) return;
        if (sparse) mc_sparse_get_results(s, E.data(), a.data(), p.data());
        else mc_get_results(d, E.data(), a.data(), p.data());
        for (int t = 0; t < NT - 1; t++)
            for (int r = 0; r < nr; r++) {
                int pa = perm[t * nr + r], pb = perm[(t + 1) * nr + r];
                double delta = (bs[t] - bs[t + 1]) * (E[pa] - E[pb]);
                bool acc = delta >= 0.0;
                if (!acc) acc = drand48() < exp(delta);
                if (acc) { perm[t * nr + r] = pb; perm[(t + 1) * nr + r] = pa; }
            }
        for (int t = 0; t < NT; t++)
            for (int r = 0; r < nr; r++) betas[perm[t * nr + r]] = bs[t];
        if (sparse) mc_sparse_set_betas(s, betas.data()); else mc_set_betas(d, betas.data());
    };
    for (int w = 0; w < warmup; w++) step();
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0);
    for (int k = 0; k < sweeps; k++) step();
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    double moves = (double)R * (N / 2) * sweeps;
    printf("%d %d %d %d %.6f %.6f %.6e\n", N, NT, nr, sweeps, ms, ms / sweeps, moves / (ms * 1e-3));
    if (sparse) mc_sparse_free(s); else mc_free(d);
    return 0;
}
