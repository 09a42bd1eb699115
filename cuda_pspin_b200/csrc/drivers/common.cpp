// common.cpp -- the reference's command-line drivers rebuilt on the C ABI.
//
// Same flags, same output directory names (config.h:65-85) and the same
// files, byte for byte in format, so the reference's analysis_pt /
// analysis_sa read them unchanged:
//   params.txt, energy_accept.txt, exchanges.txt, energy_split.txt,
//   configs.bin, temperatures.txt, frequencies.txt (FMC), quartets.txt
//   (sparse), time.txt (parallel_tempering.cu:119-176, 243-271, 355-416,
//   494-505; parallel_tempering_sparse.cu:277-296, 509-516).
// The sweep/exchange cycle between two saves runs on the device
// (pspin_pt_run); the host wakes only to write files.
//
// Extension (no reference counterpart): -batch K runs K disorder samples
// (labels label..label+K-1, seeds seed..seed+K-1) in one batched engine and
// writes one data directory per sample, as K separate runs would.
// -shard r/n runs only the samples of those K that pspin_shard_samples gives
// to shard r of n (one process per GPU, with -dev), so n processes together
// write the K directories of the unsharded run, file for file.
#include "common.h"

#include <sys/stat.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

namespace {

// "-shard r/n": r in [0, n); the indices of the K samples of shard r
bool parse_shard(const char* a, int& r, int& n) {
    return sscanf(a, "%d/%d", &r, &n) == 2 && n >= 1 && r >= 0 && r < n;
}

std::vector<int> shard_indices(int K, int N, int R, int r, int n) {
    std::vector<int> Ns(K, N), Rs(K, R), of(K, 0), mine;
    if (n > 1 && pspin_shard_samples(K, Ns.data(), Rs.data(), n, of.data()) != PSPIN_OK) return mine;
    for (int k = 0; k < K; k++)
        if (of[k] == r) mine.push_back(k);
    return mine;
}

// config.h:50-57
void fmt_param(char* buf, int sz, double v) {
    snprintf(buf, sz, "%.6g", v);
    if (!strchr(buf, '.') && !strchr(buf, 'e')) {
        int n = (int)strlen(buf);
        if (n + 3 < sz) { buf[n] = '.'; buf[n + 1] = '0'; buf[n + 2] = '\0'; }
    }
}

// config.h:65-85
void make_run_dir(char* buf, int sz, const char* base, const char* prefix, int N, double alpha, double J,
                  double J0, double alpha0, int NT, int nrep, int label) {
    char sa[32], sR[32], sa0[32];
    fmt_param(sa, sizeof(sa), alpha);
    fmt_param(sa0, sizeof(sa0), alpha0);
    if (J0 == 0.0) snprintf(sR, sizeof(sR), "inf");
    else fmt_param(sR, sizeof(sR), J / J0);
    if (label >= 0) snprintf(buf, sz, "%s/%s_N%d_a%s_R%s_a0%s_NT%d_NR%d_S%d", base, prefix, N, sa, sR, sa0, NT, nrep, label);
    else snprintf(buf, sz, "%s/%s_N%d_a%s_R%s_a0%s_NT%d_NR%d", base, prefix, N, sa, sR, sa0, NT, nrep);
}

double now_s() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + t.tv_nsec * 1e-9;
}

bool check(int rc) {
    if (rc != PSPIN_OK) {
        fprintf(stderr, "%s\n", pspin_last_error());
        return false;
    }
    return true;
}

struct SampleFiles {
    std::string dir;
    FILE* fout = nullptr;
    FILE* fex = nullptr;
    FILE* fes = nullptr;
    FILE* fconf = nullptr;
    std::vector<long long> ex_acc_last, ex_prop_last;
    void close() {
        for (FILE* f : {fout, fex, fes, fconf})
            if (f) fclose(f);
        fout = fex = fes = fconf = nullptr;
    }
};

}  // namespace

int pt_main(int argc, char** argv, int variant) {
    const bool sparse = variant == PSPIN_SPARSE;
    // parallel_tempering.cu:34-56: PT flags, the rest for parse_args
    double Tmax = -1.0, Tmin = -1.0;
    int NT = -1, pt_freq = -1, log_temp = 0, batch = 1, shard = 0, nshards = 1;
    std::vector<char*> rest;
    rest.push_back(argv[0]);
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "-Tmax") && i + 1 < argc) Tmax = atof(argv[++i]);
        else if (!strcmp(argv[i], "-Tmin") && i + 1 < argc) Tmin = atof(argv[++i]);
        else if (!strcmp(argv[i], "-NT") && i + 1 < argc) NT = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-pt_freq") && i + 1 < argc) pt_freq = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-log_temp")) log_temp = 1;
        else if (!strcmp(argv[i], "-batch") && i + 1 < argc) batch = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-shard") && i + 1 < argc) {
            if (!parse_shard(argv[++i], shard, nshards)) {
                fprintf(stderr, "Error: -shard takes r/n with 0 <= r < n\n");
                return 1;
            }
        } else rest.push_back(argv[i]);
    }
    if (Tmax < 0 || Tmin < 0 || NT < 2 || pt_freq < 1) {
        fprintf(stderr, "%s requires: -Tmax t -Tmin t -NT nt -pt_freq p\n",
                sparse ? "Sparse PT" : "Parallel Tempering");
        fprintf(stderr, "Usage: %s -N n -Tmax t -Tmin t -NT nt -pt_freq p -iter k "
                        "[-nrep n] [-J j] [-seed s] [-save_freq f] [-label l] [-dev d] "
                        "[-fmc 0|1|2] [-gamma g] [-verbose [0|1|2]] [-log_temp] [-batch K] [-shard r/n]\n",
                argv[0]);
        return 1;
    }
    if (Tmin > Tmax) {
        fprintf(stderr, "Error: Tmin (%.4f) > Tmax (%.4f)\n", Tmin, Tmax);
        return 1;
    }
    if (batch < 1) {
        fprintf(stderr, "Error: -batch must be >= 1\n");
        return 1;
    }
    pspin_config cfg;
    if (pspin_parse_args((int)rest.size(), rest.data(), &cfg) != PSPIN_OK) {
        fprintf(stderr, "%s\n", pspin_last_error());
        return 1;
    }
    const int nrep_per_temp = cfg.nrep;
    const int total_replicas = NT * nrep_per_temp;
    cfg.nrep = total_replicas;
    cfg.T = Tmax;

    // temperature schedule (parallel_tempering.cu:93-109)
    std::vector<double> T(NT), beta(NT);
    if (log_temp) {
        const double A = (NT > 1) ? pow(Tmin / Tmax, 1.0 / (NT - 1)) : 1.0;
        for (int t = 0; t < NT; t++) { T[t] = Tmax * pow(A, t); beta[t] = 1.0 / T[t]; }
    } else {
        const double dT = (NT > 1) ? (Tmax - Tmin) / (NT - 1) : 0.0;
        for (int t = 0; t < NT; t++) { T[t] = Tmax - t * dT; beta[t] = 1.0 / T[t]; }
    }

    const int label0 = (cfg.label >= 0) ? cfg.label : 0;
    const bool labelled = batch > 1 || cfg.label >= 0;
    const std::vector<int> idx = shard_indices(batch, cfg.N, total_replicas, shard, nshards);
    if (idx.empty()) {
        printf("  shard %d/%d holds none of the %d samples\n", shard, nshards, batch);
        return 0;
    }
    batch = (int)idx.size();
    std::vector<pspin_config> cfgs(batch, cfg);
    std::vector<SampleFiles> files(batch);
    mkdir("data", 0755);
    for (int k = 0; k < batch; k++) {
        cfgs[k].seed = cfg.seed + (uint64_t)idx[k];
        cfgs[k].label = labelled ? label0 + idx[k] : cfg.label;
        const int label = label0 + idx[k];
        char datadir[256];
        make_run_dir(datadir, sizeof(datadir), "data", sparse ? "PTS" : "PT", cfg.N, cfg.alpha, cfg.J, cfg.J0,
                     cfg.alpha0, NT, nrep_per_temp, label);
        mkdir(datadir, 0755);
        SampleFiles& f = files[k];
        f.dir = datadir;
        FILE* fp = fopen((f.dir + "/params.txt").c_str(), "w");
        if (fp) {
            fprintf(fp, "N %d\n", cfg.N);
            fprintf(fp, "J %.10g\n", cfg.J);
            fprintf(fp, "J0 %.10g\n", cfg.J0);
            fprintf(fp, "alpha %.10g\n", cfg.alpha);
            fprintf(fp, "alpha0 %.10g\n", cfg.alpha0);
            fprintf(fp, "NT %d\n", NT);
            fprintf(fp, "nrep %d\n", nrep_per_temp);
            fprintf(fp, "label %d\n", label);
            fprintf(fp, "seed %lu\n", (unsigned long)cfgs[k].seed);
            fprintf(fp, "nsweeps %d\n", cfg.mc_iterations);
            fprintf(fp, "Tmin %.10g\n", Tmin);
            fprintf(fp, "Tmax %.10g\n", Tmax);
            fclose(fp);
        }
        f.fout = fopen((f.dir + "/energy_accept.txt").c_str(), "w");
        f.fex = fopen((f.dir + "/exchanges.txt").c_str(), "w");
        f.fes = fopen((f.dir + "/energy_split.txt").c_str(), "w");
        if (!f.fout || !f.fex || !f.fes) {
            fprintf(stderr, "Cannot open output files\n");
            return 2;
        }
        f.fconf = fopen((f.dir + "/configs.bin").c_str(), "wb");
        if (!f.fconf) {
            fprintf(stderr, "Cannot open configs.bin\n");
            return 2;
        }
        const int hdr[3] = {cfg.N, NT, nrep_per_temp};
        fwrite(hdr, sizeof(int), 3, f.fconf);
        fprintf(f.fout, "# sweep\tTidx\tT");
        for (int r = 0; r < nrep_per_temp; r++) fprintf(f.fout, "\tE%d/N\tacc%d", r, r);
        fprintf(f.fout, "\n");
        fprintf(f.fex, "# sweep\tTidx\tT_high\tT_low\tn_acc\tn_prop\trate\n");
        fprintf(f.fes, "# sweep\tTidx\tT");
        for (int r = 0; r < nrep_per_temp; r++) fprintf(f.fes, "\tE2_%d/N\tE4_%d/N", r, r);
        fprintf(f.fes, "\n");
        f.ex_acc_last.assign(NT - 1, 0);
        f.ex_prop_last.assign(NT - 1, 0);
    }

    printf("\n  p-Spin 2+4 :: %s (B200 engine)\n", sparse ? "Sparse Parallel Tempering" : "Parallel Tempering");
    pspin_options opt;
    memset(&opt, 0, sizeof(opt));
    opt.trace_replica = -1;
    pspin_state* st = nullptr;
    if (!check(pspin_create_batch(cfgs.data(), batch, variant, &opt, &st))) return 1;

    const int N = cfg.N;
    for (int k = 0; k < batch; k++) {
        SampleFiles& f = files[k];
        pspin_info info;
        if (!check(pspin_get_info(st, k, &info))) return 1;
        if (cfg.fmc_mode > 0) {
            const char* names[] = {"FC", "comb", "uniform"};
            printf("  %-22s %s (gamma=%.6f)  pairs=%lld/%lld  quartets=%lld/%lld\n", "FMC active",
                   names[cfg.fmc_mode], cfg.gamma, (long long)info.n_pairs_active, (long long)N * (N + 1) / 2,
                   (long long)info.n_quart_active, (long long)N * (N - 1) * (N - 2) * (N - 3) / 24);
            std::vector<double> w(N);
            if (!check(pspin_get_omega(st, k, w.data()))) return 1;
            FILE* ff = fopen((f.dir + "/frequencies.txt").c_str(), "w");
            if (ff) {
                fprintf(ff, "# i omega_i\n");
                for (int i = 0; i < N; i++) fprintf(ff, "%d\t%.12f\n", i, w[i]);
                fclose(ff);
            }
        }
        if (sparse) {
            std::vector<int32_t> q((size_t)info.n_quartets * 5);
            std::vector<double> g(info.n_quartets);
            if (!check(pspin_get_sparse_quartets(st, k, q.data(), g.data()))) return 1;
            FILE* fsq = fopen((f.dir + "/quartets.txt").c_str(), "w");
            if (fsq) {
                fprintf(fsq, "# idx i j k l ch Re(g)\n");
                for (int s = 0; s < info.n_quartets; s++)
                    fprintf(fsq, "%d\t%d\t%d\t%d\t%d\t%d\t%.12e\n", s, q[5 * s], q[5 * s + 1], q[5 * s + 2],
                            q[5 * s + 3], q[5 * s + 4], g[s]);
                fclose(fsq);
            }
        }
        FILE* ft = fopen((f.dir + "/temperatures.txt").c_str(), "w");
        if (ft) {
            fprintf(ft, "# Tidx T beta\n");
            for (int t = 0; t < NT; t++) fprintf(ft, "%d\t%.12f\t%.12f\n", t, T[t], beta[t]);
            fclose(ft);
        }
    }
    if (!check(pspin_pt_init(st, NT, nrep_per_temp, beta.data(), pt_freq))) return 1;

    const int R_all = batch * total_replicas;
    std::vector<double> E(R_all), e2(R_all), e4(R_all), spins((size_t)R_all * N * 2);
    std::vector<int64_t> acc(R_all), prop(R_all);
    std::vector<int32_t> perm(total_replicas);
    std::vector<int64_t> exa(NT - 1), exp_(NT - 1);
    std::vector<int64_t> ex_total_acc((size_t)batch * (NT - 1)), ex_total_prop((size_t)batch * (NT - 1));

    const double t_start = now_s();
    int s = 0;
    while (s < cfg.mc_iterations) {
        // next save point: (s+1) % save_freq == 0 or the last sweep
        int next = s;
        while (!((next + 1) % cfg.save_freq == 0 || next == cfg.mc_iterations - 1)) next++;
        if (!check(pspin_pt_run(st, next - s + 1))) return 1;
        s = next;
        if (!check(pspin_get_results(st, E.data(), acc.data(), prop.data()))) return 1;
        if (!check(pspin_split_energies(st, e2.data(), e4.data()))) return 1;
        const bool save_conf = s >= cfg.mc_iterations / 2;
        if (save_conf && !check(pspin_get_spins(st, spins.data()))) return 1;
        for (int k = 0; k < batch; k++) {
            SampleFiles& f = files[k];
            const int off = k * total_replicas;
            if (!check(pspin_pt_get(st, k, perm.data(), exa.data(), exp_.data()))) return 1;
            // energy & acceptance per temperature (:359-369), window rates since the last save
            for (int t = 0; t < NT; t++) {
                fprintf(f.fout, "%d\t%d\t%.8f", s + 1, t, T[t]);
                for (int r = 0; r < nrep_per_temp; r++) {
                    const int phys = off + perm[t * nrep_per_temp + r];
                    const double a = (prop[phys] > 0) ? (double)acc[phys] / prop[phys] : 0.0;
                    fprintf(f.fout, "\t%.8f\t%.5f", E[phys] / N, a);
                }
                fprintf(f.fout, "\n");
            }
            fflush(f.fout);
            // exchange rates, window since the last save (:372-381)
            for (int t = 0; t < NT - 1; t++) {
                const long long wa = exa[t] - f.ex_acc_last[t], wp = exp_[t] - f.ex_prop_last[t];
                const double rate = (wp > 0) ? (double)wa / wp : 0.0;
                fprintf(f.fex, "%d\t%d\t%.8f\t%.8f\t%lld\t%lld\t%.5f\n", s + 1, t, T[t], T[t + 1], wa, wp, rate);
                f.ex_acc_last[t] = exa[t];
                f.ex_prop_last[t] = exp_[t];
                ex_total_acc[(size_t)k * (NT - 1) + t] = exa[t];
                ex_total_prop[(size_t)k * (NT - 1) + t] = exp_[t];
            }
            fflush(f.fex);
            // split energies (:384-393)
            for (int t = 0; t < NT; t++) {
                fprintf(f.fes, "%d\t%d\t%.8f", s + 1, t, T[t]);
                for (int r = 0; r < nrep_per_temp; r++) {
                    const int phys = off + perm[t * nrep_per_temp + r];
                    fprintf(f.fes, "\t%.8f\t%.8f", e2[phys] / N, e4[phys] / N);
                }
                fprintf(f.fes, "\n");
            }
            fflush(f.fes);
            // configurations in the second half, logical (t, r) order (:400-416)
            if (save_conf) {
                const int sweep = s + 1;
                fwrite(&sweep, sizeof(int), 1, f.fconf);
                for (int t = 0; t < NT; t++)
                    for (int r = 0; r < nrep_per_temp; r++) {
                        const int phys = off + perm[t * nrep_per_temp + r];
                        fwrite(&spins[(size_t)phys * N * 2], sizeof(double), 2 * (size_t)N, f.fconf);
                    }
                fflush(f.fconf);
            }
            if (cfg.verbose == 1 && k == 0) {
                const int cold = perm[(NT - 1) * nrep_per_temp], hot = perm[0];
                printf("  sweep %d/%d:  E_hot/N=% .3e  E_cold/N=% .3e\n", s + 1, cfg.mc_iterations, E[hot] / N,
                       E[cold] / N);
            }
        }
        if (!check(pspin_reset_counters(st))) return 1;   // :396-397
        s++;
    }
    const double elapsed = now_s() - t_start;
    printf("\n  %-22s %.3f s\n", "total time", elapsed);
    printf("  %-22s %.4f ms\n", "time/sweep", elapsed / cfg.mc_iterations * 1e3);
    printf("  %-22s %d\n", "sweeps", cfg.mc_iterations);
    printf("  %-22s %d\n", "total replicas", total_replicas);
    printf("  %-22s %d\n", "samples", batch);
    for (int t = 0; t < NT - 1; t++) {
        const long long a = ex_total_acc[t], p = ex_total_prop[t];
        printf("  T[%d]-T[%d]  (%.4f-%.4f)  %lld/%lld = %.4f\n", t, t + 1, T[t], T[t + 1], a, p,
               p > 0 ? (double)a / p : 0.0);
    }
    for (int k = 0; k < batch; k++) {
        SampleFiles& f = files[k];
        FILE* ftim = fopen((f.dir + "/time.txt").c_str(), "w");
        if (ftim) {
            pspin_info info;
            pspin_get_info(st, k, &info);
            if (sparse) {
                fprintf(ftim, "# N NT nrep_per_temp total_replicas mc_iterations pt_freq save_freq Tmax Tmin n_sparse "
                              "total_time_s ms_per_sweep\n");
                fprintf(ftim, "%d %d %d %d %d %d %d %.6f %.6f %d %.6f %.6f\n", N, NT, nrep_per_temp, total_replicas,
                        cfg.mc_iterations, pt_freq, cfg.save_freq, Tmax, Tmin, info.n_quartets, elapsed,
                        elapsed / cfg.mc_iterations * 1e3);
            } else {
                fprintf(ftim, "# N NT nrep_per_temp total_replicas mc_iterations pt_freq save_freq Tmax Tmin "
                              "total_time_s ms_per_sweep\n");
                fprintf(ftim, "%d %d %d %d %d %d %d %.6f %.6f %.6f %.6f\n", N, NT, nrep_per_temp, total_replicas,
                        cfg.mc_iterations, pt_freq, cfg.save_freq, Tmax, Tmin, elapsed,
                        elapsed / cfg.mc_iterations * 1e3);
            }
            fclose(ftim);
        }
        f.close();
    }
    pspin_destroy(st);
    return 0;
}

int sa_main(int argc, char** argv) {
    // simulated_annealing.cu:32-70: SA flags, the rest for parse_args
    double Tmax = -1.0, Tmin = -1.0;
    int ntemp = -1, batch = 1, shard = 0, nshards = 1;
    std::vector<char*> rest;
    rest.push_back(argv[0]);
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "-Tmax") && i + 1 < argc) Tmax = atof(argv[++i]);
        else if (!strcmp(argv[i], "-Tmin") && i + 1 < argc) Tmin = atof(argv[++i]);
        else if (!strcmp(argv[i], "-ntemp") && i + 1 < argc) ntemp = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-batch") && i + 1 < argc) batch = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-shard") && i + 1 < argc) {
            if (!parse_shard(argv[++i], shard, nshards)) {
                fprintf(stderr, "Error: -shard takes r/n with 0 <= r < n\n");
                return 1;
            }
        } else rest.push_back(argv[i]);
    }
    if (Tmax < 0 || Tmin < 0 || ntemp < 1) {
        fprintf(stderr, "Simulated Annealing requires: -Tmax tmax -Tmin tmin -ntemp nt\n");
        fprintf(stderr, "Usage: %s -N n -Tmax tmax -Tmin tmin -ntemp nt -iter k "
                        "[-nrep n] [-J j] [-seed s] [-save_freq f] [-label l] [-dev d] "
                        "[-fmc 0|1|2] [-gamma g] [-verbose [0|1|2]] [-batch K] [-shard r/n]\n", argv[0]);
        return 1;
    }
    if (Tmin > Tmax) {
        fprintf(stderr, "Error: Tmin (%.4f) > Tmax (%.4f)\n", Tmin, Tmax);
        return 1;
    }
    if (batch < 1) {
        fprintf(stderr, "Error: -batch must be >= 1\n");
        return 1;
    }
    pspin_config cfg;
    if (pspin_parse_args((int)rest.size(), rest.data(), &cfg) != PSPIN_OK) {
        fprintf(stderr, "%s\n", pspin_last_error());
        return 1;
    }
    if (cfg.mc_iterations < 0 || cfg.mc_iterations > 30) {
        fprintf(stderr, "Error: -iter k gives 2^k sweeps per temperature; k must be in [0, 30]\n");
        return 1;
    }
    const int sweeps_per_temp = 1 << cfg.mc_iterations;    // :72
    const int N = cfg.N, nrep = cfg.nrep;
    cfg.T = Tmax;                                           // :173

    // one data directory per sample, data/SA_N{N}_NR{nrep}_S{label} (:83-100)
    const int label0 = (cfg.label >= 0) ? cfg.label : 0;
    const std::vector<int> idx = shard_indices(batch, N, nrep, shard, nshards);
    if (idx.empty()) {
        printf("  shard %d/%d holds none of the %d samples\n", shard, nshards, batch);
        return 0;
    }
    batch = (int)idx.size();
    std::vector<pspin_config> cfgs(batch, cfg);
    std::vector<std::string> dirs(batch);
    std::vector<FILE*> fouts(batch, nullptr);
    mkdir("data", 0755);
    for (int k = 0; k < batch; k++) {
        cfgs[k].seed = cfg.seed + (uint64_t)idx[k];
        cfgs[k].label = label0 + idx[k];
        char datadir[256];
        snprintf(datadir, sizeof(datadir), "data/SA_N%d_NR%d_S%d", N, nrep, label0 + idx[k]);
        mkdir(datadir, 0755);
        dirs[k] = datadir;
        mkdir((dirs[k] + "/configs").c_str(), 0755);
        fouts[k] = fopen((dirs[k] + "/energy_accept.txt").c_str(), "w");
        if (!fouts[k]) {
            fprintf(stderr, "Cannot open %s/energy_accept.txt\n", datadir);
            return 2;
        }
        fprintf(fouts[k], "# T\tsweep");
        for (int r = 0; r < nrep; r++) fprintf(fouts[k], "\tE%d/N\tacc%d", r, r);
        fprintf(fouts[k], "\n");
    }

    printf("\n  p-Spin 2+4 :: Simulated Annealing (B200 engine)\n");
    pspin_options opt;
    memset(&opt, 0, sizeof(opt));
    opt.trace_replica = -1;
    pspin_state* st = nullptr;
    if (!check(pspin_create_batch(cfgs.data(), batch, PSPIN_DENSE, &opt, &st))) return 1;
    if (cfg.fmc_mode > 0) {                                 // :176-194
        for (int k = 0; k < batch; k++) {
            std::vector<double> w(N);
            if (!check(pspin_get_omega(st, k, w.data()))) return 1;
            FILE* ff = fopen((dirs[k] + "/frequencies.txt").c_str(), "w");
            if (ff) {
                fprintf(ff, "# i omega_i\n");
                for (int i = 0; i < N; i++) fprintf(ff, "%d\t%.12f\n", i, w[i]);
                fclose(ff);
            }
        }
    }

    const int R_all = batch * nrep;
    std::vector<double> E(R_all), spins((size_t)R_all * N * 2);
    std::vector<int64_t> acc(R_all), prop(R_all);
    const double t0 = now_s();
    // geometric cooling T_k = Tmax A^k, A = (Tmin/Tmax)^(1/(ntemp-1)) (:207-208, :218-220)
    const double A = (ntemp > 1) ? pow(Tmin / Tmax, 1.0 / (ntemp - 1)) : 1.0;
    printf("  %-22s %.8f\n", "schedule (A)", A);
    for (int step = 0; step < ntemp; step++) {
        const double T = Tmax * pow(A, step);
        // mc_sweep refills every beta with 1/T before each sweep (mc.cu:749-752);
        // T is fixed within a step, so one fill per step is the same
        if (!check(pspin_fill_betas(st, 1.0 / T))) return 1;
        if (!check(pspin_reset_counters(st))) return 1;     // :223-224
        int s = 0;
        while (s < sweeps_per_temp) {
            int next = s;
            while (!((next + 1) % cfg.save_freq == 0 || next == sweeps_per_temp - 1)) next++;
            if (!check(pspin_sweep(st, next - s + 1))) return 1;
            s = next;
            if (!check(pspin_get_results(st, E.data(), acc.data(), prop.data()))) return 1;
            for (int k = 0; k < batch; k++) {               // :238-246
                fprintf(fouts[k], "%.8f\t%d", T, s + 1);
                for (int r = 0; r < nrep; r++) {
                    const int i = k * nrep + r;
                    const double a = (prop[i] > 0) ? (double)acc[i] / prop[i] : 0.0;
                    fprintf(fouts[k], "\t%.8f\t%.5f", E[i] / N, a);
                }
                fprintf(fouts[k], "\n");
                fflush(fouts[k]);
            }
            if (!check(pspin_reset_counters(st))) return 1; // :268-270
            s++;
        }
        if (step >= ntemp / 2) {                            // :274-292
            if (!check(pspin_get_spins(st, spins.data()))) return 1;
            for (int k = 0; k < batch; k++)
                for (int r = 0; r < nrep; r++) {
                    char conffile[512];
                    snprintf(conffile, sizeof(conffile), "%s/configs/conf_r%d_T%.6f.bin", dirs[k].c_str(), r, T);
                    FILE* fc = fopen(conffile, "wb");
                    if (fc) {
                        fwrite(&spins[(size_t)(k * nrep + r) * N * 2], sizeof(double), 2 * (size_t)N, fc);
                        fclose(fc);
                    }
                }
        }
        if (cfg.verbose == 1) {
            printf("  [%d/%d] T=%.6f", step + 1, ntemp, T);
            for (int r = 0; r < nrep; r++) printf("  E/N=%.4f", E[r] / N);
            printf("\n");
        }
    }
    const double elapsed = now_s() - t0;
    printf("\n  %-22s %.3f s\n", "total time", elapsed);
    printf("  %-22s %d x %d = %lld\n", "total sweeps", ntemp, sweeps_per_temp, (long long)ntemp * sweeps_per_temp);
    printf("  %-22s %d\n", "samples", batch);
    for (int k = 0; k < batch; k++) {                       // :307-315
        FILE* ftim = fopen((dirs[k] + "/time.txt").c_str(), "w");
        if (ftim) {
            fprintf(ftim, "# N nrep ntemp sweeps_per_temp Tmax Tmin total_time_s\n");
            fprintf(ftim, "%d %d %d %d %.6f %.6f %.6f\n", N, nrep, ntemp, sweeps_per_temp, Tmax, Tmin, elapsed);
            fclose(ftim);
        }
        fclose(fouts[k]);
    }
    pspin_destroy(st);
    return 0;
}

int mc_main(int argc, char** argv) {
    pspin_config cfg;
    if (pspin_parse_args(argc, argv, &cfg) != PSPIN_OK) {
        fprintf(stderr, "%s\n", pspin_last_error());
        return 1;
    }
    // montecarlo.cu:39-60
    char datadir[128];
    if (cfg.label >= 0) snprintf(datadir, sizeof(datadir), "data/N%d_NR%d_S%d", cfg.N, cfg.nrep, cfg.label);
    else snprintf(datadir, sizeof(datadir), "data/N%d_NR%d", cfg.N, cfg.nrep);
    mkdir("data", 0755);
    mkdir(datadir, 0755);
    std::string confdir = std::string(datadir) + "/configs";
    mkdir(confdir.c_str(), 0755);
    FILE* fout = fopen((std::string(datadir) + "/energy_accept.txt").c_str(), "w");
    if (!fout) {
        fprintf(stderr, "Cannot open %s/energy_accept.txt\n", datadir);
        return 2;
    }
    fprintf(fout, "# iter");
    for (int r = 0; r < cfg.nrep; r++) fprintf(fout, "\tE%d/N\tacc%d", r, r);
    fprintf(fout, "\n");
    pspin_options opt;
    memset(&opt, 0, sizeof(opt));
    opt.trace_replica = -1;
    pspin_state* st = nullptr;
    if (!check(pspin_create(&cfg, PSPIN_DENSE, &opt, &st))) return 1;
    const int N = cfg.N;
    if (cfg.fmc_mode > 0) {
        std::vector<double> w(N);
        if (!check(pspin_get_omega(st, 0, w.data()))) return 1;
        FILE* ff = fopen((std::string(datadir) + "/frequencies.txt").c_str(), "w");
        if (ff) {
            fprintf(ff, "# i omega_i\n");
            for (int i = 0; i < N; i++) fprintf(ff, "%d\t%.12f\n", i, w[i]);
            fclose(ff);
        }
    }
    if (!check(pspin_fill_betas(st, 1.0 / cfg.T))) return 1;   // mc_sweep's fill (mc.cu:752)
    std::vector<double> E(cfg.nrep), spins((size_t)cfg.nrep * N * 2);
    std::vector<int64_t> acc(cfg.nrep), prop(cfg.nrep);
    const double t0 = now_s();
    int s = 0;
    while (s < cfg.mc_iterations) {
        int next = s;
        while (!((next + 1) % cfg.save_freq == 0 || next == cfg.mc_iterations - 1)) next++;
        if (!check(pspin_sweep(st, next - s + 1))) return 1;
        s = next;
        if (!check(pspin_get_results(st, E.data(), acc.data(), prop.data()))) return 1;
        fprintf(fout, "%d", s + 1);
        for (int r = 0; r < cfg.nrep; r++) {
            const double a = (prop[r] > 0) ? (double)acc[r] / prop[r] : 0.0;
            fprintf(fout, "\t%.8f\t%.5f", E[r] / N, a);
        }
        fprintf(fout, "\n");
        fflush(fout);
        if (s >= cfg.mc_iterations / 2) {
            if (!check(pspin_get_spins(st, spins.data()))) return 1;
            for (int r = 0; r < cfg.nrep; r++) {
                char conffile[512];
                snprintf(conffile, sizeof(conffile), "%s/conf_r%d_iter%d.bin", confdir.c_str(), r, s + 1);
                FILE* fc = fopen(conffile, "wb");
                if (fc) {
                    fwrite(&spins[(size_t)r * N * 2], sizeof(double), 2 * (size_t)N, fc);
                    fclose(fc);
                }
            }
        }
        s++;
    }
    const double elapsed = now_s() - t0;
    const double t_per_iter = elapsed / cfg.mc_iterations;
    printf("\n  %-22s %.3f s\n  %-22s %.4f ms\n", "total time", elapsed, "time/sweep", t_per_iter * 1e3);
    FILE* ftim = fopen((std::string(datadir) + "/time_per_iter.txt").c_str(), "w");
    if (ftim) {
        fprintf(ftim, "# N nrep mc_iterations total_time_s ms_per_iter\n");
        fprintf(ftim, "%d %d %d %.6f %.6f\n", N, cfg.nrep, cfg.mc_iterations, elapsed, t_per_iter * 1e3);
        fclose(ftim);
    }
    fclose(fout);
    pspin_destroy(st);
    return 0;
}
