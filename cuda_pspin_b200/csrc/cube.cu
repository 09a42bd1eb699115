// cube.cu -- the smoothed-cube check of the reference (smoothed_cube.cu) on
// the engine: many independent configurations projected onto
// sum_k |a_k|^4 = N, and a free walk (no Hamiltonian: every move accepted)
// of one configuration with the engine's FP32 cube proposal.
#include "sweep_common.cuh"

namespace pspin {

// One thread per configuration: scale every amplitude by
// (N / sum_k |a_k|^4)^(1/4), the sum in site order in FP64, as the
// reference's normalize_many_cube_kernel does (smoothed_cube.cu:52-66).
__global__ void cube_normalize_many_kernel(double* all, int N, int nsamples) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsamples) return;
    double* sp = all + (size_t)s * 2 * N;
    double sum_r4 = 0.0;
    for (int i = 0; i < N; i++) {
        const double re = sp[2 * i], im = sp[2 * i + 1];
        const double r2 = re * re + im * im;
        sum_r4 += r2 * r2;
    }
    const double scale = pow((double)N / sum_r4, 0.25);
    for (int i = 0; i < 2 * N; i++) sp[i] *= scale;
}

cudaError_t launch_cube_normalize_many(double* all, int N, int nsamples, cudaStream_t st) {
    if (nsamples <= 0) return cudaSuccess;
    cube_normalize_many_kernel<<<(nsamples + 255) / 256, 256, 0, st>>>(all, N, nsamples);
    return cudaGetLastError();
}

// One thread walks one configuration: N/2 pair moves per sweep (the pair
// (0,1) when N = 2, otherwise the engine's pair pick), each the engine's
// cube proposal (propose<1>) from the walk's counter-based streams, always
// accepted; the state is saved (FP64 from the FP32 amplitudes) before the
// first sweep and after every save_freq-th, up to max_saved records.
__global__ void cube_walk_kernel(float2* a, int N, int sweeps, int save_freq, uint32_t k0, uint32_t k1,
                                 uint32_t p0, uint32_t p1, double* traj, int max_saved, int* n_saved) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int saved = 0;
    auto save = [&]() {
        if (saved >= max_saved) return;
        for (int k = 0; k < N; k++) {
            traj[((size_t)saved * N + k) * 2] = (double)a[k].x;
            traj[((size_t)saved * N + k) * 2 + 1] = (double)a[k].y;
        }
        saved++;
    };
    save();
    const int steps = N / 2 > 0 ? N / 2 : 1;
    for (int sw = 0; sw < sweeps; sw++) {
        for (int p = 0; p < steps; p++) {
            int i0 = 0, j0 = 1;
            if (N > 2) pair_pick(p0, p1, (uint64_t)sw, (uint32_t)p, N, i0, j0);
            float2 ain, ajn;
            propose<1>(a[i0], a[j0], move_words(k0, k1, (uint64_t)sw, (uint32_t)p), ain, ajn);
            a[i0] = ain;
            a[j0] = ajn;
        }
        if ((sw + 1) % save_freq == 0) save();
    }
    *n_saved = saved;
}

cudaError_t launch_cube_walk(float2* a, int N, int sweeps, int save_freq, uint64_t move_key, uint64_t pair_key,
                             double* traj, int max_saved, int* n_saved, cudaStream_t st) {
    cube_walk_kernel<<<1, 1, 0, st>>>(a, N, sweeps, save_freq, (uint32_t)move_key, (uint32_t)(move_key >> 32),
                                      (uint32_t)pair_key, (uint32_t)(pair_key >> 32), traj, max_saved, n_saved);
    return cudaGetLastError();
}

}  // namespace pspin
