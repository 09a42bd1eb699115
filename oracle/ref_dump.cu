// ref_dump.cu -- test harness linked against the reference's own objects
// (built by oracle/Makefile into oracle/_ref/ref_dump; runs on a GPU).
//
// Calls the reference's mc_init / mc_sparse_init (mc.cu:411-562,
// mc_sparse.cu:390-604) for one configuration and writes its state as raw
// little-endian arrays into an output directory, so that tests can compare
// the engine and the oracle against the reference's actual numbers:
//   info.txt        N nrep fmc gamma n_pairs_active n_quart_active h2_active n_quartets
//   g2.f64          N*N complex     (dense and sparse)
//   g4.f64, mask.u8 C(N,4)          (dense only)
//   quartets.txt    i j k l ch g    (sparse only, %.17g)
//   omega.f64       N               (fmc > 0)
//   spins.f64       nrep*N complex  initial amplitudes
//   energies.f64    nrep            initial energies (chain form)
//   after.f64 / after_E.f64         spins and running energies after -sweeps
//                                   sweeps at beta = 1/T (optional)
//
// usage: ref_dump <outdir> dense|sparse [reference flags: -N -nrep -seed -fmc -gamma -J -alpha ...]
//        [-sweeps k]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "config.h"
#include "disorder.h"
#include "mc.h"
#include "mc_sparse.h"

static void dump(const std::string& path, const void* p, size_t bytes) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    fwrite(p, 1, bytes, f);
    fclose(f);
}

int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s outdir dense|sparse [flags]\n", argv[0]); return 1; }
    std::string out = argv[1];
    bool sparse = !strcmp(argv[2], "sparse");
    int sweeps = 0;
    std::vector<char*> rest;
    rest.push_back(argv[0]);
    for (int i = 3; i < argc; i++) {
        if (!strcmp(argv[i], "-sweeps") && i + 1 < argc) sweeps = atoi(argv[++i]);
        else rest.push_back(argv[i]);
    }
    SimConfig cfg = parse_args((int)rest.size(), rest.data());
    const int N = cfg.N, R = cfg.nrep;
    std::vector<double> betas(R, 1.0 / cfg.T);
    std::vector<cuDoubleComplex> spins((size_t)R * N);
    std::vector<double> E(R);
    std::vector<long long> acc(R), prop(R);
    FILE* fi = fopen((out + "/info.txt").c_str(), "w");
    if (!sparse) {
        MCState s = mc_init(cfg);
        long long nq = n_quartets(N);
        std::vector<cuDoubleComplex> g2((size_t)N * N), g4(nq);
        std::vector<unsigned char> mask(nq);
        cudaMemcpy(g2.data(), s.d_g2, g2.size() * sizeof(cuDoubleComplex), cudaMemcpyDeviceToHost);
        cudaMemcpy(g4.data(), s.d_g4, g4.size() * sizeof(cuDoubleComplex), cudaMemcpyDeviceToHost);
        cudaMemcpy(mask.data(), s.d_g4_mask, mask.size(), cudaMemcpyDeviceToHost);
        dump(out + "/g2.f64", g2.data(), g2.size() * sizeof(cuDoubleComplex));
        dump(out + "/g4.f64", g4.data(), g4.size() * sizeof(cuDoubleComplex));
        dump(out + "/mask.u8", mask.data(), mask.size());
        if (s.h_omega) dump(out + "/omega.f64", s.h_omega, N * sizeof(double));
        mc_get_spins(s, spins.data());
        mc_get_results(s, E.data(), acc.data(), prop.data());
        dump(out + "/spins.f64", spins.data(), spins.size() * sizeof(cuDoubleComplex));
        dump(out + "/energies.f64", E.data(), E.size() * sizeof(double));
        fprintf(fi, "%d %d %d %.17g %lld %lld %d %d\n", N, R, cfg.fmc_mode, cfg.gamma, s.n_pairs_active,
                s.n_quart_active, s.h2_active, 0);
        if (sweeps > 0) {
            mc_set_betas(s, betas.data());
            for (int k = 0; k < sweeps; k++) mc_sweep_pt(s);
            mc_get_spins(s, spins.data());
            mc_get_results(s, E.data(), acc.data(), prop.data());
            dump(out + "/after.f64", spins.data(), spins.size() * sizeof(cuDoubleComplex));
            dump(out + "/after_E.f64", E.data(), E.size() * sizeof(double));
        }
        mc_free(s);
    } else {
        MCStateSparse s = mc_sparse_init(cfg);
        std::vector<cuDoubleComplex> g2((size_t)N * N);
        cudaMemcpy(g2.data(), s.d_g2, g2.size() * sizeof(cuDoubleComplex), cudaMemcpyDeviceToHost);
        dump(out + "/g2.f64", g2.data(), g2.size() * sizeof(cuDoubleComplex));
        std::vector<SparseQuartet> q(s.n_quartets);
        cudaMemcpy(q.data(), s.d_quartets, q.size() * sizeof(SparseQuartet), cudaMemcpyDeviceToHost);
        FILE* fq = fopen((out + "/quartets.txt").c_str(), "w");
        for (size_t t = 0; t < q.size(); t++)
            fprintf(fq, "%d %d %d %d %d %.17g\n", q[t].i, q[t].j, q[t].k, q[t].l, q[t].ch, q[t].g.x);
        fclose(fq);
        if (s.h_omega) dump(out + "/omega.f64", s.h_omega, N * sizeof(double));
        mc_sparse_get_spins(s, spins.data());
        mc_sparse_get_results(s, E.data(), acc.data(), prop.data());
        dump(out + "/spins.f64", spins.data(), spins.size() * sizeof(cuDoubleComplex));
        dump(out + "/energies.f64", E.data(), E.size() * sizeof(double));
        fprintf(fi, "%d %d %d %.17g %lld %lld %d %d\n", N, R, cfg.fmc_mode, cfg.gamma, s.n_pairs_active,
                s.n_quart_active, s.h2_active, s.n_quartets);
        if (sweeps > 0) {
            mc_sparse_set_betas(s, betas.data());
            for (int k = 0; k < sweeps; k++) mc_sparse_sweep_pt(s);
            mc_sparse_get_spins(s, spins.data());
            mc_sparse_get_results(s, E.data(), acc.data(), prop.data());
            dump(out + "/after.f64", spins.data(), spins.size() * sizeof(cuDoubleComplex));
            dump(out + "/after_E.f64", E.data(), E.size() * sizeof(double));
        }
        mc_sparse_free(s);
    }
    fclose(fi);
    return 0;
}
