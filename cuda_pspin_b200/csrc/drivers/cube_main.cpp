// pspin_smoothed_cube: the reference's smoothed_cube check (smoothed_cube.cu)
// on the engine.  Same flags and data files in smoothed_cube/:
//   init_scatter.dat, moduli.dat   nsamples configurations on
//                                  sum |a_k|^4 = N (pspin_cube_samples: the
//                                  reference's cuRAND stream and scaling);
//   squircle.dat, superellipse.dat the analytic boundaries;
//   mc_trajectory.dat              a free walk (no Hamiltonian) with the
//                                  engine's cube move (pspin_cube_walk).
// The gnuplot scripts and images the reference also writes are not made.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <vector>

#include "pspin.h"

static void write_squircle(const char* fname, int N, int npts) {
    FILE* f = fopen(fname, "w");
    if (!f) { perror(fname); return; }
    const double s = pow((double)N, 0.25);
    fprintf(f, "# Squircle boundary: |x|^4 + |y|^4 = %d\n", N);
    for (int i = 0; i <= npts; i++) {
        const double t = 2.0 * M_PI * i / npts;
        const double ct = cos(t), st = sin(t);
        fprintf(f, "%.8f %.8f\n", (ct >= 0 ? 1.0 : -1.0) * s * sqrt(fabs(ct)), (st >= 0 ? 1.0 : -1.0) * s * sqrt(fabs(st)));
    }
    fclose(f);
}

static void write_superellipse(const char* fname, int N, int npts) {
    FILE* f = fopen(fname, "w");
    if (!f) { perror(fname); return; }
    const double s = pow((double)N, 0.25);
    fprintf(f, "# Superellipse: r1^4 + r2^4 = %d  (first quadrant)\n", N);
    for (int i = 0; i <= npts; i++) {
        const double t = 0.5 * M_PI * i / npts;
        fprintf(f, "%.8f %.8f\n", s * sqrt(cos(t)), s * sqrt(sin(t)));
    }
    fclose(f);
}

static int check(int rc) {
    if (rc != PSPIN_OK) {
        fprintf(stderr, "pspin: %s\n", pspin_last_error());
        exit(1);
    }
    return rc;
}

int main(int argc, char** argv) {
    int N = 2, iter = 10, nsamples = 10000;
    unsigned long long seed = 42;
    for (int i = 1; i < argc; i++) {
        if (strcmp(argv[i], "-N") == 0 && i + 1 < argc) N = atoi(argv[++i]);
        else if (strcmp(argv[i], "-iter") == 0 && i + 1 < argc) iter = atoi(argv[++i]);
        else if (strcmp(argv[i], "-seed") == 0 && i + 1 < argc) seed = strtoull(argv[++i], nullptr, 10);
        else if (strcmp(argv[i], "-nsamples") == 0 && i + 1 < argc) nsamples = atoi(argv[++i]);
        else {
            fprintf(stderr, "Usage: %s [-N 2] [-iter 10] [-seed 42] [-nsamples 10000]\n", argv[0]);
            exit(1);
        }
    }
    if (N < 2) {
        fprintf(stderr, "Error: N must be >= 2.\n");
        exit(1);
    }
    if (iter < 0 || iter > 30 || nsamples < 1) {
        fprintf(stderr, "Error: need 0 <= iter <= 30 and nsamples >= 1.\n");
        exit(1);
    }
    const int sweeps = 1 << iter;
    const int save_freq = (sweeps > 2048) ? sweeps / 1024 : 1;
    printf("  N        = %d\n  sweeps   = %d  (2^%d)\n  seed     = %llu\n  nsamples = %d\n"
           "  save_freq= %d  (~%d trajectory points)\n\n",
           N, sweeps, iter, seed, nsamples, save_freq, sweeps / save_freq + 1);
    if (mkdir("smoothed_cube", 0755) != 0 && errno != EEXIST) {
        perror("smoothed_cube");
        return 1;
    }

    std::vector<double> all(2 * (size_t)N * nsamples);
    check(pspin_cube_samples(N, nsamples, seed, all.data()));
    {
        FILE* f = fopen("smoothed_cube/init_scatter.dat", "w");
        if (!f) { perror("smoothed_cube/init_scatter.dat"); return 1; }
        fprintf(f, "# Re(a_1)  Re(a_2)\n");
        for (int s = 0; s < nsamples; s++)
            fprintf(f, "%.8f %.8f\n", all[(size_t)s * 2 * N], all[(size_t)s * 2 * N + 2]);
        fclose(f);
    }
    {
        FILE* f = fopen("smoothed_cube/moduli.dat", "w");
        if (!f) { perror("smoothed_cube/moduli.dat"); return 1; }
        fprintf(f, "# |a_1|  |a_2|\n");
        for (int s = 0; s < nsamples; s++) {
            const double* a = &all[(size_t)s * 2 * N];
            fprintf(f, "%.8f %.8f\n", sqrt(a[0] * a[0] + a[1] * a[1]), sqrt(a[2] * a[2] + a[3] * a[3]));
        }
        fclose(f);
    }
    write_squircle("smoothed_cube/squircle.dat", N, 1000);
    write_superellipse("smoothed_cube/superellipse.dat", N, 500);
    printf("  Written smoothed_cube/init_scatter.dat, moduli.dat, squircle.dat, superellipse.dat\n");

    const int max_saved = sweeps / save_freq + 2;
    std::vector<double> traj(2 * (size_t)N * max_saved);
    int n_saved = 0;
    check(pspin_cube_walk(N, sweeps, save_freq, seed, traj.data(), max_saved, &n_saved));
    FILE* f = fopen("smoothed_cube/mc_trajectory.dat", "w");
    if (!f) { perror("smoothed_cube/mc_trajectory.dat"); return 1; }
    fprintf(f, "# sweep  Re(a1)  Re(a2)  |a1|  |a2|  S4\n");
    for (int i = 0; i < n_saved; i++) {
        const double* a = &traj[(size_t)i * 2 * N];
        double S4 = 0.0;
        for (int k = 0; k < N; k++) {
            const double rk = sqrt(a[2 * k] * a[2 * k] + a[2 * k + 1] * a[2 * k + 1]);
            S4 += rk * rk * rk * rk;
        }
        fprintf(f, "%d %.8f %.8f %.8f %.8f %.15f\n", i == 0 ? 0 : i * save_freq, a[0], a[2],
                sqrt(a[0] * a[0] + a[1] * a[1]), sqrt(a[2] * a[2] + a[3] * a[3]), S4);
    }
    fclose(f);
    printf("  Written smoothed_cube/mc_trajectory.dat (%d points)\n", n_saved);
    return 0;
}
