// mlp.cuh -- the learned pair-move proposal: a small MLP over the pair's
// local-field features that outputs a Beta law for the amplitude transfer
// t' = |a_i'|^2 / (|a_i|^2 + |a_j|^2) and one 4-component von Mises mixture
// per site for the new phase measured from the site's field,
// psi = theta' + arg(h).  Densities, samplers and the loss gradient.
//
// Plain move (spins.h:17-52) in the same coordinates: t' ~ Beta(1/2, 1/2)
// (t' = cos^2 alpha, alpha uniform) and uniform phases, independent of the
// state.  The plain chain with acceptance min(1, e^{-beta dE}) samples
// e^{-beta E} nu with nu ~ Beta(1/2,1/2)(t) (the measure its proposal is
// symmetric for); a learned proposal keeps that target with
//   A = min(1, e^{-beta dE} [q_L(x|x')/q_P(x|x')] / [q_L(x'|x)/q_P(x'|x)]).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>
#include "rng.cuh"

namespace pspin {

constexpr int kMlpIn = 8, kMlpHidden = 64, kMlpOut = 26;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHidden;
constexpr int kMlpParams = kOffB3 + kMlpOut;                 // 6426
constexpr int kRecordFloats = kMlpIn + 3;                    // features, t', psi_i, psi_j
constexpr float kKappaMax = 50.0f;
constexpr float kTEdge = 1e-7f;          // the learned move's t' lies in (kTEdge, 1 - kTEdge)
constexpr float kTwoPi = 6.283185307179586f;

// Features of a pair at one state: log(1+beta sqrt(S)|h|) for both sites,
// cos/sin of each site's phase measured from its field, 2t-1, log(beta).
__device__ __forceinline__ void pair_features(float2 ai, float2 aj, float2 hi, float2 hj, float beta, float* f) {
    const float ri = fmaf(ai.x, ai.x, ai.y * ai.y), rj = fmaf(aj.x, aj.x, aj.y * aj.y);
    const float S = ri + rj, sS = sqrtf(S);
    const float mi = sqrtf(fmaf(hi.x, hi.x, hi.y * hi.y)), mj = sqrtf(fmaf(hj.x, hj.x, hj.y * hj.y));
    f[0] = log1pf(beta * sS * mi);
    f[1] = log1pf(beta * sS * mj);
    const float pi = atan2f(ai.y, ai.x) + atan2f(hi.y, hi.x);
    const float pj = atan2f(aj.y, aj.x) + atan2f(hj.y, hj.x);
    float s, c;
    sincosf(pi, &s, &c);
    f[2] = c; f[3] = s;
    sincosf(pj, &s, &c);
    f[4] = c; f[5] = s;
    f[6] = 2.0f * ri / S - 1.0f;
    f[7] = logf(beta > 1e-30f ? beta : 1e-30f);
}

// Forward pass of one record with FP32 weights; the hidden activations go to
// the record's rows h1[64], h2[64] (which the backward pass reads) and are
// read back from there.  (A variant holding them in per-thread arrays gave
// wrong outputs for the second site's mixture under nvcc 12.9 -O3; this form
// is checked against float64 autograd.)
__device__ __forceinline__ void mlp_forward_rows(const float* __restrict__ w, const float* f, float* h1, float* h2,
                                                 float* out) {
    for (int o = 0; o < kMlpHidden; o++) {
        float z = w[kOffB1 + o];
#pragma unroll
        for (int i = 0; i < kMlpIn; i++) z = fmaf(w[kOffW1 + o * kMlpIn + i], f[i], z);
        h1[o] = tanhf(z);
    }
    for (int o = 0; o < kMlpHidden; o++) {
        float z = w[kOffB2 + o];
        for (int i = 0; i < kMlpHidden; i++) z = fmaf(w[kOffW2 + o * kMlpHidden + i], h1[i], z);
        h2[o] = tanhf(z);
    }
    for (int o = 0; o < kMlpOut; o++) {
        float z = w[kOffB3 + o];
        for (int i = 0; i < kMlpHidden; i++) z = fmaf(w[kOffW3 + o * kMlpHidden + i], h2[i], z);
        out[o] = z;
    }
}

__device__ __forceinline__ float softplusf(float x) { return x > 20.f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

struct ProposalParams {
    float a, b;               // Beta(a, b) for t'
    float w[2][4], mu[2][4], kappa[2][4];   // mixtures for psi_i, psi_j
};

__device__ __forceinline__ float decode_beta_param(float o) { return 0.05f + softplusf(o); }

// one site's mixture from its 12 outputs q: softmax weights, means, kappas
__device__ __forceinline__ void decode_site(const float* q, float* w, float* mu, float* kappa) {
    float m = q[0];
    #pragma unroll
    for (int k = 1; k < 4; k++) m = fmaxf(m, q[k]);
    float z = 0.f;
    #pragma unroll
    for (int k = 0; k < 4; k++) { w[k] = expf(q[k] - m); z += w[k]; }
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        w[k] /= z;
        mu[k] = q[4 + k];
        kappa[k] = kKappaMax * sigmoidf(q[8 + k]) + 0.01f;
    }
}

__device__ __forceinline__ void decode_outputs(const float* o, ProposalParams& p) {
    p.a = decode_beta_param(o[0]);
    p.b = decode_beta_param(o[1]);
    #pragma unroll
    for (int s = 0; s < 2; s++) decode_site(o + 2 + 12 * s, p.w[s], p.mu[s], p.kappa[s]);
}

// log I0(k) for 0 < k <= kKappaMax (CUDA's Bessel function, no overflow there)
__device__ __forceinline__ float log_i0f(float k) { return logf(cyl_bessel_i0f(k)); }

// log Beta(a,b) density at t with the log-gamma values given
__device__ __forceinline__ float log_beta_pdf_lg(float t, float a, float b, float lga, float lgb, float lgab) {
    return (a - 1.0f) * logf(t) + (b - 1.0f) * log1pf(-t) - (lga + lgb - lgab);
}

__device__ __forceinline__ float log_beta_pdf(float t, float a, float b) {
    return log_beta_pdf_lg(t, a, b, lgammaf(a), lgammaf(b), lgammaf(a + b));
}

// log of the plain proposal density in (t', theta_i', theta_j'):
// Beta(1/2,1/2)(t) / (2 pi)^2
__device__ __forceinline__ float log_plain_density(float t) {
    return -0.5f * logf(t) - 0.5f * log1pf(-t) - 1.1447298858494002f - 2.0f * 1.8378770664093453f;
}

__device__ __forceinline__ float log_vm_mix_site(const float* w, const float* mu, const float* kappa, float psi) {
    float m = -1e30f, v[4];
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = logf(w[k]) + kappa[k] * cosf(psi - mu[k]) - 1.8378770664093453f - log_i0f(kappa[k]);
        m = fmaxf(m, v[k]);
    }
    float z = 0.f;
    #pragma unroll
    for (int k = 0; k < 4; k++) z += expf(v[k] - m);
    return m + logf(z);
}

__device__ __forceinline__ float log_vm_mix(const ProposalParams& p, int s, float psi) {
    return log_vm_mix_site(p.w[s], p.mu[s], p.kappa[s], psi);
}

__device__ __forceinline__ float log_learned_density(const ProposalParams& p, float t, float psi_i, float psi_j) {
    return log_beta_pdf(t, p.a, p.b) + log_vm_mix(p, 0, psi_i) + log_vm_mix(p, 1, psi_j);
}

// ------------------------------------------------------------------ sampling
// A counter-based stream of uniforms for one replica's move: Philox blocks
// (key, {step, sweep, tag + n}) drawn four words at a time.
struct MoveStream {
    uint32_t k0, k1, step, sw_lo, sw_hi, n, used;
    U4 w;
    __device__ __forceinline__ uint32_t next() {
        if (used == 4) {
            w = philox4x32_10(U4{step, sw_lo, sw_hi, 0x6c726e00u + n}, k0, k1);
            n++;
            used = 0;
        }
        const uint32_t v = used == 0 ? w.x : used == 1 ? w.y : used == 2 ? w.z : w.w;
        used++;
        return v;
    }
    __device__ __forceinline__ float uniform() { return u01f_open0(next()); }   // (0, 1]
};

__device__ __forceinline__ float normal(MoveStream& g) {
    const float u1 = g.uniform(), u2 = g.uniform();
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Marsaglia & Tsang (2000) gamma sampler, bounded; returns < 0 on exhaustion
__device__ __forceinline__ float gamma_sample(MoveStream& g, float a) {
    float boost = 1.0f;
    if (a < 1.0f) {
        boost = powf(g.uniform(), 1.0f / a);
        a += 1.0f;
    }
    const float d = a - 1.0f / 3.0f, c = rsqrtf(9.0f * d);
    for (int it = 0; it < 32; it++) {
        const float x = normal(g);
        float v = 1.0f + c * x;
        if (v <= 0.0f) continue;
        v = v * v * v;
        const float u = g.uniform();
        if (logf(u) < 0.5f * x * x + d - d * v + d * logf(v)) return d * v * boost;
    }
    return -1.0f;
}

// Best & Fisher (1979) von Mises sampler around 0, bounded; -10 on exhaustion
__device__ __forceinline__ float vonmises_sample(MoveStream& g, float kappa) {
    if (kappa < 1e-3f) return kTwoPi * g.uniform() - 3.14159265f;
    const float tau = 1.0f + sqrtf(1.0f + 4.0f * kappa * kappa);
    const float rho = (tau - sqrtf(2.0f * tau)) / (2.0f * kappa);
    const float r = (1.0f + rho * rho) / (2.0f * rho);
    for (int it = 0; it < 32; it++) {
        const float u1 = g.uniform(), u2 = g.uniform();
        const float z = cospif(u1);
        const float f = (1.0f + r * z) / (r + z);
        const float c = kappa * (r - f);
        if (c * (2.0f - c) - u2 > 0.0f || logf(c / u2) + 1.0f - c >= 0.0f) {
            const float th = acosf(fminf(1.0f, fmaxf(-1.0f, f)));
            return g.uniform() < 0.5f ? -th : th;
        }
    }
    return -10.0f;
}

// component k of a 4-component mixture for a uniform u by an unrolled scan
// (constant indices keep the parameters in registers); returns its kappa, mu
__device__ __forceinline__ void pick_component(const float* w, const float* mu, const float* kappa, float u,
                                               float& kap, float& m) {
    float acc = w[0];
    kap = kappa[0];
    m = mu[0];
    bool done = u <= acc;
#pragma unroll
    for (int k = 1; k < 4; k++) {
        if (!done) { kap = kappa[k]; m = mu[k]; }
        acc += w[k];
        done = done || u <= acc;
    }
}

// ---- the learned move split in five independent roles ----------------------
// Given the network outputs, the move's four random parts are independent:
// t' = X/(X+Y) with X ~ Gamma(a), Y ~ Gamma(b), and each site's phase from
// its own mixture.  Each role runs one of them as a complete rejection
// sampler on its own sub-stream of the replica's move stream (Philox blocks
// kRoleBlocks*r ..), so the roles can run on different warps at once and the
// draw is still exact; the density's parts (log-gamma values, each site's
// mixture log-density at its phase) go with them.  Role 4 takes lgamma(a+b).
// Results go to rows of a [kXchRows][32] exchange buffer (lane = replica).
constexpr int kRoles = 5;
constexpr uint32_t kRoleBlocks = 40;               // >= 25 blocks a bounded gamma or von Mises draw can use
constexpr uint32_t kAcceptBlock = kRoles * kRoleBlocks;   // the accept (and record) draws
enum : int { X_A, X_B, X_X, X_Y, X_LGA, X_LGB, X_LGAB, X_PSI0, X_PSI1, X_VM0, X_VM1, X_OK0, X_OK1, kXchRows };

__device__ __forceinline__ MoveStream role_stream(uint32_t k0, uint32_t k1, uint32_t step, uint64_t sw,
                                                  uint32_t first_block) {
    return MoveStream{k0, k1, step, (uint32_t)sw, (uint32_t)(sw >> 32), first_block, 4u, U4{0u, 0u, 0u, 0u}};
}

// out(o) reads output o of this lane's replica.  sample: forward move (draw
// and density parts); otherwise the reverse density's parts at the phases
// already in rows X_PSI0 / X_PSI1.
template <class Out>
__device__ __forceinline__ void learned_role(int r, bool sample, Out out, float* xch, int lane, uint32_t k0,
                                             uint32_t k1, uint32_t step, uint64_t sw) {
    if (r < 2) {
        const float a = decode_beta_param(out(r));
        xch[(X_A + r) * 32 + lane] = a;
        xch[(X_LGA + r) * 32 + lane] = lgammaf(a);
        if (sample) {
            MoveStream g = role_stream(k0, k1, step, sw, kRoleBlocks * (uint32_t)r);
            xch[(X_X + r) * 32 + lane] = gamma_sample(g, a);
        }
    } else if (r < 4) {
        const int s = r - 2;
        float q[12], w[4], mu[4], kap[4];
#pragma unroll
        for (int o = 0; o < 12; o++) q[o] = out(2 + 12 * s + o);
        decode_site(q, w, mu, kap);
        float psi = sample ? 0.0f : xch[(X_PSI0 + s) * 32 + lane];
        bool ok = true;
        if (sample) {
            MoveStream g = role_stream(k0, k1, step, sw, kRoleBlocks * (uint32_t)r);
            float kk, mm;
            pick_component(w, mu, kap, g.uniform(), kk, mm);
            const float v = vonmises_sample(g, kk);
            ok = v >= -9.0f;
            psi = mm + v;
            xch[(X_PSI0 + s) * 32 + lane] = psi;
            xch[(X_OK0 + s) * 32 + lane] = ok ? 1.0f : 0.0f;
        }
        xch[(X_VM0 + s) * 32 + lane] = ok ? log_vm_mix_site(w, mu, kap, psi) : 0.0f;
    } else {
        xch[X_LGAB * 32 + lane] = lgammaf(decode_beta_param(out(0)) + decode_beta_param(out(1)));
    }
}

// ------------------------------------------------------------------ training
// digamma by recurrence to x >= 6 and the asymptotic series
// (Abramowitz & Stegun 6.3.18)
__device__ __forceinline__ float digammaf_series(float x) {
    float r = 0.f;
    while (x < 6.0f) { r -= 1.0f / x; x += 1.0f; }
    const float i2 = 1.0f / (x * x);
    return r + logf(x) - 0.5f / x - i2 * (1.0f / 12.0f - i2 * (1.0f / 120.0f - i2 / 252.0f));
}

// d(-log q_L)/d(outputs) for one record; returns -log q_L
__device__ __forceinline__ float loss_output_grad(const float* o, float t, float psi_i, float psi_j, float* g) {
    ProposalParams p;
    decode_outputs(o, p);
    float loss = -log_learned_density(p, t, psi_i, psi_j);
    const float dab = digammaf_series(p.a + p.b);
    g[0] = -(logf(t) - digammaf_series(p.a) + dab) * sigmoidf(o[0]);
    g[1] = -(log1pf(-t) - digammaf_series(p.b) + dab) * sigmoidf(o[1]);
    const float psis[2] = {psi_i, psi_j};
    #pragma unroll
    for (int s = 0; s < 2; s++) {
        const float* q = o + 2 + 12 * s;
        float* gq = g + 2 + 12 * s;
        float v[4], m = -1e30f;
        #pragma unroll
        for (int k = 0; k < 4; k++) {
            v[k] = logf(p.w[s][k]) + p.kappa[s][k] * cosf(psis[s] - p.mu[s][k]) - log_i0f(p.kappa[s][k]);
            m = fmaxf(m, v[k]);
        }
        float z = 0.f;
        #pragma unroll
        for (int k = 0; k < 4; k++) { v[k] = expf(v[k] - m); z += v[k]; }
        #pragma unroll
        for (int k = 0; k < 4; k++) {
            const float rk = v[k] / z;          // responsibility
            const float kap = p.kappa[s][k], dpsi = psis[s] - p.mu[s][k];
            gq[k] = p.w[s][k] - rk;
            gq[4 + k] = -rk * kap * sinf(dpsi);
            const float ratio = cyl_bessel_i1f(kap) / cyl_bessel_i0f(kap);
            const float sg = sigmoidf(q[8 + k]);
            gq[8 + k] = -rk * (cosf(dpsi) - ratio) * kKappaMax * sg * (1.0f - sg);
        }
    }
    return loss;
}

}  // namespace pspin
