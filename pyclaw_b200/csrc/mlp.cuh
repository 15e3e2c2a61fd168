// mlp.cuh -- the learned Newton guess of the exact Euler solver.
//
// Network: 6 -> 32 -> 32 -> 1, tanh hidden layers, linear output; inputs and
// output as in exact_euler::features (the guess is p0 * exp(w * y), p0 the
// adaptive PVRS guess, w = J^2/(1+J^2) a jump weight, so a weak wave keeps the
// accurate PVRS value).  Parameters (FP32, 1313): W1[32][6], b1[32],
// W2[32][32], b2[32], W3[32], b3.
//
// Training (all kernels of this file, FP32): k_gen_samples draws seeded
// Riemann problems and solves each to tol by FP64 Newton; k_train_grad runs
// forward and backward for a minibatch (one sample per thread, gradients
// reduced per warp with shuffles, then atomically added); k_adam applies Adam.
//
// Inference: k_mlp_guess_tc, one thread per grid site, evaluates the MLP for
// the x- and y-interface of the site (interfaces with a weak jump keep the
// PVRS guess) in BF16 on the tensor cores with FP32 accumulation --
// tcgen05.mma from shared-memory operands into TMEM accumulators, 128
// interfaces per MMA tile -- and writes the guesses that the step kernel's
// Newton iteration starts from.  k_mlp_guess is the same pass on the
// warp-level mma.sync.m16n8k16 (64 interfaces = 4 row tiles per warp; a
// layer's accumulator fragments are exactly the next layer's A fragments),
// kept as the comparison path (claw2_mlp_set_engine).
#pragma once

#include <cuda_bf16.h>

#include "riemann.cuh"

namespace claw2 {

constexpr int MLP_IN = 6, MLP_H = 32;
// Jump weight below which the learned correction is not applied (J^2 < 0.053).
constexpr double MLP_WMIN = 0.05;
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1;  // 1313
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + MLP_H * MLP_IN, OFF_W2 = OFF_B1 + MLP_H,
              OFF_B2 = OFF_W2 + MLP_H * MLP_H, OFF_W3 = OFF_B2 + MLP_H, OFF_B3 = OFF_W3 + MLP_H;

// ---- counter-based random numbers (splitmix64 finaliser of seed ^ index) ----
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ double u01(unsigned long long seed, unsigned long long i, int k) {
    const unsigned long long z = mix64(seed ^ mix64(i * 8ull + (unsigned long long)k));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
}

// The training distribution: rho, p log-uniform in [1e-2, 1e2], u uniform in
// [-3, 3] on both sides.
__host__ __device__ __forceinline__ void draw_problem(unsigned long long seed, unsigned long long i, double& rl,
                                                      double& ul, double& pl, double& rr, double& ur, double& pr) {
    const double l10 = 2.302585092994046;
    rl = exp(l10 * (-2.0 + 4.0 * u01(seed, i, 0)));
    pl = exp(l10 * (-2.0 + 4.0 * u01(seed, i, 1)));
    ul = -3.0 + 6.0 * u01(seed, i, 2);
    rr = exp(l10 * (-2.0 + 4.0 * u01(seed, i, 3)));
    pr = exp(l10 * (-2.0 + 4.0 * u01(seed, i, 4)));
    ur = -3.0 + 6.0 * u01(seed, i, 5);
}

// x[i*8 + 0..5] features, x[i*8+6] = jump weight w, y[i] target, ok[i] = 0 for vacuum.
static __global__ void k_gen_samples(unsigned long long seed, long long first, int n, double gamma, double tol,
                                     float* x, float* y, int* ok, double* pstar) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const unsigned long long i = (unsigned long long)(first + k);
    double rl, ul, pl, rr, ur, pr;
    draw_problem(seed, i, rl, ul, pl, rr, ur, pr);
    const exact_euler::Gas G = exact_euler::make_gas(gamma);
    const double cl = sqrt(gamma * pl / rl), cr = sqrt(gamma * pr / rr);
    float f[6];
    double w;
    exact_euler::features(G, rl, ul, pl, rr, ur, pr, f, w);
    for (int j = 0; j < 6; ++j) x[(long long)k * 8 + j] = f[j];
    x[(long long)k * 8 + 6] = (float)w;
    x[(long long)k * 8 + 7] = 0.f;
    if (exact_euler::vacuum(G, ul, cl, ur, cr)) {
        ok[k] = 0;
        y[k] = 0.f;
        if (pstar) pstar[k] = 0.0;
        return;
    }
    double ps, us;
    int it;
    exact_euler::star(G, rl, ul, pl, cl, rr, ur, pr, cr, 0.0, tol, 200, ps, us, it);
    const double p0 = exact_euler::guess_pvrs(G, rl, ul, pl, cl, rr, ur, pr, cr);
    const bool good = ps > 0.0 && p0 > 0.0 && w > 1e-12;
    ok[k] = good ? 1 : 0;
    y[k] = good ? (float)(log(ps / p0) / w) : 0.f;
    if (pstar) pstar[k] = ps;
}

// FP32 forward pass for one sample (training and the reference evaluation).
__device__ __forceinline__ float mlp_forward(const float* P, const float (&x)[6], float (&h1)[MLP_H],
                                             float (&h2)[MLP_H]) {
#pragma unroll 4
    for (int j = 0; j < MLP_H; ++j) {
        float z = P[OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < 6; ++i) z = fmaf(P[OFF_W1 + j * 6 + i], x[i], z);
        h1[j] = tanhf(z);
    }
#pragma unroll 4
    for (int j = 0; j < MLP_H; ++j) {
        float z = P[OFF_B2 + j];
#pragma unroll 8
        for (int i = 0; i < MLP_H; ++i) z = fmaf(P[OFF_W2 + j * MLP_H + i], h1[i], z);
        h2[j] = tanhf(z);
    }
    float out = P[OFF_B3];
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) out = fmaf(P[OFF_W3 + i], h2[i], out);
    return out;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Gradient of 0.5 * mean squared error over samples [first, first+count);
// grad (MLP_NPARAM floats) and loss are accumulated (caller zeroes them).
static __global__ void __launch_bounds__(256) k_train_grad(const float* __restrict__ P, const float* __restrict__ x,
                                                           const float* __restrict__ y, const int* __restrict__ ok,
                                                           long long first, int count, float inv_n, float* grad,
                                                           float* loss) {
    __shared__ float sP[MLP_NPARAM];
    __shared__ float sG[MLP_NPARAM];
    for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) {
        sP[k] = P[k];
        sG[k] = 0.f;
    }
    __syncthreads();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = k < count && ok[first + k];
    float xi[6], h1[MLP_H], h2[MLP_H];
    const long long s = first + (act ? k : 0);
#pragma unroll
    for (int i = 0; i < 6; ++i) xi[i] = x[s * 8 + i];
    const float out = mlp_forward(sP, xi, h1, h2);
    const float e = act ? (out - y[s]) : 0.f;
    const float dy = e * inv_n;
    // output layer
    {
        const float g = warp_sum(dy);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_B3], g);
    }
    float dz2[MLP_H];
#pragma unroll 4
    for (int j = 0; j < MLP_H; ++j) {
        const float g = warp_sum(dy * h2[j]);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_W3 + j], g);
        dz2[j] = dy * sP[OFF_W3 + j] * (1.f - h2[j] * h2[j]);
    }
    // second hidden layer
#pragma unroll 2
    for (int j = 0; j < MLP_H; ++j) {
        const float gb = warp_sum(dz2[j]);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_B2 + j], gb);
        for (int i = 0; i < MLP_H; ++i) {
            const float g = warp_sum(dz2[j] * h1[i]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_W2 + j * MLP_H + i], g);
        }
    }
    // first hidden layer
#pragma unroll 2
    for (int i = 0; i < MLP_H; ++i) {
        float d = 0.f;
        for (int j = 0; j < MLP_H; ++j) d = fmaf(sP[OFF_W2 + j * MLP_H + i], dz2[j], d);
        const float dz1 = d * (1.f - h1[i] * h1[i]);
        const float gb = warp_sum(dz1);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_B1 + i], gb);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float g = warp_sum(dz1 * xi[c]);
            if ((threadIdx.x & 31) == 0) atomicAdd(&sG[OFF_W1 + i * 6 + c], g);
        }
    }
    const float l = warp_sum(0.5f * e * e * inv_n);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
    __syncthreads();
    for (int q = threadIdx.x; q < MLP_NPARAM; q += blockDim.x) atomicAdd(&grad[q], sG[q]);
}

// Adam (Kingma & Ba 2015); zeroes the gradient afterwards.
static __global__ void k_adam(float* P, float* grad, float* m, float* v, float lr, float b1, float b2, float eps,
                              int step) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float mh = mk / (1.f - powf(b1, (float)step));
    const float vh = vk / (1.f - powf(b2, (float)step));
    P[k] -= lr * mh / (sqrtf(vh) + eps);
    grad[k] = 0.f;
}

// ---- BF16 tensor-core inference ---------------------------------------------
// Inference weights: B fragments of each layer in the mma.sync layout, made
// from the FP32 parameters on the host side of this file (mlp_pack).
struct MlpPacked {
    unsigned int w1[4][32][2];     // layer 1: 4 n-tiles (K = 16: 6 inputs + zeros)
    unsigned int w2[4][2][32][2];  // layer 2: 4 n-tiles x 2 k-tiles
    unsigned int w3[2][32][2];     // layer 3: 1 n-tile (column 0) x 2 k-tiles
    float b1[MLP_H], b2[MLP_H], b3;
};

__host__ __device__ __forceinline__ unsigned short bf16_bits(float f) {
    // round-to-nearest-even conversion of an FP32 value to BF16 bits
    unsigned int u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (unsigned short)((u >> 16) | ((u & 0xffff) ? 0x40 : 0));
    u += 0x7fffu + ((u >> 16) & 1u);
    return (unsigned short)(u >> 16);
}
__host__ __device__ __forceinline__ unsigned int pack2(float lo, float hi) {
    return (unsigned int)bf16_bits(lo) | ((unsigned int)bf16_bits(hi) << 16);
}

// Fill the fragments (host): B[k][n] = W[n][k]; lane = 4g + t holds
// (k = 2t, 2t+1; n = g) in register 0 and (k = 2t+8, 2t+9; n = g) in register 1.
inline void mlp_pack(const float* P, MlpPacked& M) {
    auto w1 = [&](int n, int k) { return k < 6 ? P[OFF_W1 + n * 6 + k] : 0.f; };
    auto w2 = [&](int n, int k) { return P[OFF_W2 + n * MLP_H + k]; };
    auto w3 = [&](int n, int k) { return n == 0 ? P[OFF_W3 + k] : 0.f; };
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, t = lane & 3;
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * j + g;
            M.w1[j][lane][0] = pack2(w1(n, 2 * t), w1(n, 2 * t + 1));
            M.w1[j][lane][1] = pack2(w1(n, 2 * t + 8), w1(n, 2 * t + 9));
            for (int kk = 0; kk < 2; ++kk) {
                M.w2[j][kk][lane][0] = pack2(w2(n, 16 * kk + 2 * t), w2(n, 16 * kk + 2 * t + 1));
                M.w2[j][kk][lane][1] = pack2(w2(n, 16 * kk + 2 * t + 8), w2(n, 16 * kk + 2 * t + 9));
            }
        }
        for (int kk = 0; kk < 2; ++kk) {
            M.w3[kk][lane][0] = pack2(w3(g, 16 * kk + 2 * t), w3(g, 16 * kk + 2 * t + 1));
            M.w3[kk][lane][1] = pack2(w3(g, 16 * kk + 2 * t + 8), w3(g, 16 * kk + 2 * t + 9));
        }
    }
    for (int j = 0; j < MLP_H; ++j) {
        M.b1[j] = P[OFF_B1 + j];
        M.b2[j] = P[OFF_B2 + j];
    }
    M.b3 = P[OFF_B3];
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned int (&a)[4], unsigned int b0, unsigned int b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// MLP outputs for the 16 rows of one M-tile whose layer-1 A fragment is `a1`.
// Returns, in lanes with t == 0, out[0] = row g and out[1] = row g + 8.
__device__ __forceinline__ void mlp_tile(const MlpPacked& M, const unsigned int (&a1)[4], float (&out)[2]) {
    const int lane = threadIdx.x & 31, t = lane & 3;
    unsigned int a2[2][4];
    {
        float d[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float bl = M.b1[8 * j + 2 * t], bh = M.b1[8 * j + 2 * t + 1];
            d[j][0] = bl; d[j][1] = bh; d[j][2] = bl; d[j][3] = bh;
            mma_bf16(d[j], a1, M.w1[j][lane][0], M.w1[j][lane][1]);
        }
        // tanh, then the accumulators of n-tiles (2kk, 2kk+1) are layer 2's A fragment kk
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            a2[kk][0] = pack2(tanh_fast(d[2 * kk][0]), tanh_fast(d[2 * kk][1]));
            a2[kk][1] = pack2(tanh_fast(d[2 * kk][2]), tanh_fast(d[2 * kk][3]));
            a2[kk][2] = pack2(tanh_fast(d[2 * kk + 1][0]), tanh_fast(d[2 * kk + 1][1]));
            a2[kk][3] = pack2(tanh_fast(d[2 * kk + 1][2]), tanh_fast(d[2 * kk + 1][3]));
        }
    }
    unsigned int a3[2][4];
    {
        float d[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float bl = M.b2[8 * j + 2 * t], bh = M.b2[8 * j + 2 * t + 1];
            d[j][0] = bl; d[j][1] = bh; d[j][2] = bl; d[j][3] = bh;
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) mma_bf16(d[j], a2[kk], M.w2[j][kk][lane][0], M.w2[j][kk][lane][1]);
        }
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            a3[kk][0] = pack2(tanh_fast(d[2 * kk][0]), tanh_fast(d[2 * kk][1]));
            a3[kk][1] = pack2(tanh_fast(d[2 * kk][2]), tanh_fast(d[2 * kk][3]));
            a3[kk][2] = pack2(tanh_fast(d[2 * kk + 1][0]), tanh_fast(d[2 * kk + 1][1]));
            a3[kk][3] = pack2(tanh_fast(d[2 * kk + 1][2]), tanh_fast(d[2 * kk + 1][3]));
        }
    }
    float d[4] = {M.b3, 0.f, M.b3, 0.f};
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) mma_bf16(d, a3[kk], M.w3[kk][lane][0], M.w3[kk][lane][1]);
    out[0] = d[0];
    out[1] = d[2];
}

// Evaluate the network for 64 feature rows held in shared memory
// (rows[64][8] floats, 6 features used) by one warp; results to res[64].
__device__ __forceinline__ void mlp_warp64(const MlpPacked& M, const float (*rows)[8], float* res) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        const int r0 = 16 * mt + g, r1 = r0 + 8;
        auto feat = [&](int r, int c) { return c < 6 ? rows[r][c] : 0.f; };
        unsigned int a[4];
        a[0] = pack2(feat(r0, 2 * t), feat(r0, 2 * t + 1));
        a[1] = pack2(feat(r1, 2 * t), feat(r1, 2 * t + 1));
        a[2] = pack2(feat(r0, 2 * t + 8), feat(r0, 2 * t + 9));
        a[3] = pack2(feat(r1, 2 * t + 8), feat(r1, 2 * t + 9));
        float out[2];
        mlp_tile(M, a, out);
        if (t == 0) {
            res[r0] = out[0];
            res[r1] = out[1];
        }
    }
    __syncwarp();
}

// Network outputs for n feature rows (x[i*8 + 0..5]) -- the raw evaluator
// behind claw2_mlp_infer; one warp per 64 rows.
static __global__ void k_mlp_eval(const MlpPacked* __restrict__ Mg, const float* __restrict__ x, int n, float* y) {
    __shared__ MlpPacked M;
    __shared__ float rows[4][64][8];
    __shared__ float res[4][64];
    for (int k = threadIdx.x; k < (int)(sizeof(MlpPacked) / 4); k += blockDim.x)
        reinterpret_cast<unsigned int*>(&M)[k] = reinterpret_cast<const unsigned int*>(Mg)[k];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long base = ((long long)blockIdx.x * 4 + w) * 64;
    for (int r = lane; r < 64; r += 32)
        for (int c = 0; c < 8; ++c) rows[w][r][c] = (base + r < n) ? x[(base + r) * 8 + c] : 0.f;
    __syncthreads();
    mlp_warp64(M, rows[w], res[w]);
    for (int r = lane; r < 64; r += 32)
        if (base + r < n) y[base + r] = res[w][r];
}

// Learned guesses for every interface of a grid: thread (cp, R) computes the
// x-interface (cp-1 | cp) on row R and the y-interface (R-1 | R) on column cp.
// guess planes: [0] x-interfaces, [1] y-interfaces, q's layout.
static __global__ void __launch_bounds__(128) k_mlp_guess(const MlpPacked* __restrict__ Mg,
                                                          const double* __restrict__ q, Layout L, double gamma,
                                                          double* guess) {
    __shared__ MlpPacked M;
    __shared__ float rows[4][64][8];
    __shared__ float res[4][64];
    for (int k = threadIdx.x; k < (int)(sizeof(MlpPacked) / 4); k += blockDim.x)
        reinterpret_cast<unsigned int*>(&M)[k] = reinterpret_cast<const unsigned int*>(Mg)[k];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cp = blockIdx.x * 32 + lane;
    const int R = blockIdx.y * 4 + w;
    const int c = min(cp, L.mx + 3), r = min(R, L.my + 3);
    const exact_euler::Gas G = exact_euler::make_gas(gamma);
    const double g1 = gamma - 1.0;
    auto prim = [&](int cc, int rr, double& rho, double& u, double& v, double& p) {
        const long long o = (long long)rr * L.pitch + cc;
        rho = q[o];
        u = q[L.plane + o] / rho;
        v = q[2 * L.plane + o] / rho;
        p = g1 * (q[3 * L.plane + o] - 0.5 * rho * (u * u + v * v));
    };
    double r0, u0, v0, p0, rl, ul, vl, pl, rb, ub, vb, pb;
    prim(c, r, r0, u0, v0, p0);
    prim(max(c - 1, 0), r, rl, ul, vl, pl);
    prim(c, max(r - 1, 0), rb, ub, vb, pb);
    double wx, wy;
    float fx[6], fy[6];
    exact_euler::features(G, rl, ul, pl, r0, u0, p0, fx, wx);
    exact_euler::features(G, rb, vb, pb, r0, v0, p0, fy, wy);
    for (int k = 0; k < 6; ++k) {
        rows[w][lane][k] = isfinite(fx[k]) ? fx[k] : 0.f;
        rows[w][32 + lane][k] = isfinite(fy[k]) ? fy[k] : 0.f;
    }
    __syncthreads();
    // PVRS decides: a weak jump (w below MLP_WMIN) keeps the PVRS guess,
    // which is accurate there and where the network has seen no training data;
    // a warp with only weak jumps skips the network altogether.
    const bool strong = (wx >= MLP_WMIN) || (wy >= MLP_WMIN);
    if (__any_sync(0xffffffffu, strong)) {
        mlp_warp64(M, rows[w], res[w]);
    } else {
        res[w][lane] = 0.f;
        res[w][32 + lane] = 0.f;
    }
    if (wx < MLP_WMIN) wx = 0.0;
    if (wy < MLP_WMIN) wy = 0.0;
    if (cp > L.mx + 3 || R > L.my + 3) return;
    const double cl = sqrt(gamma * pl / rl), c0 = sqrt(gamma * p0 / r0), cb = sqrt(gamma * pb / rb);
    const double gx0 = exact_euler::guess_pvrs(G, rl, ul, pl, cl, r0, u0, p0, c0);
    const double gy0 = exact_euler::guess_pvrs(G, rb, vb, pb, cb, r0, v0, p0, c0);
    const long long o = (long long)R * L.pitch + cp;
    guess[o] = gx0 * exp(wx * (double)res[w][lane]);
    guess[L.plane + o] = gy0 * exp(wy * (double)res[w][32 + lane]);
}

// ---- BF16 inference on the 5th-generation tensor cores (tcgen05 + TMEM) -----
// One CTA of 128 threads evaluates the network for two M = 128 row tiles at a
// time (the x- and the y-interfaces of 128 grid sites, or 256 rows of
// features): thread t owns row t of both tiles, which is TMEM lane t of the
// accumulators, so warp w reads back exactly the lanes 32w..32w+31 it may
// access.  Per tile pair: layer 1 is one tcgen05.mma (M 128, N 32, K 16) per
// tile, the 32 FP32 accumulators of a row come back with one tcgen05.ld,
// tanh and the BF16 rounding run in registers and the row goes back to
// shared memory as layer 2's A operand; layer 2 is two K = 16 MMAs per tile
// into the same TMEM columns; layer 3 (32 -> 1) is a 32-term FP32 dot product
// of the BF16-rounded activations in each thread.  Operands are BF16 in the
// no-swizzle K-major layout of the tcgen05 shared-memory descriptors: element
// (r, k) of an R x K matrix at byte (r/8)*16K + (k/8)*128 + (r%8)*16 + (k%8)*2
// (8 x 16-byte core matrices; the leading, K, offset 128 bytes; the stride
// between 8-row groups 16K bytes).  One elected thread issues the MMAs and
// commits them to an mbarrier; every wait on it is bounded (status bit 1).
struct MlpTcImage {                  // device image of the weights, copied into shared memory
    unsigned short w1[MLP_H * 16];   // layer 1 B operand: N = 32 x K = 16 (6 inputs + zeros)
    unsigned short w2[MLP_H * MLP_H];  // layer 2 B operand: N = 32 x K = 32
    float b1[MLP_H], b2[MLP_H];
    float w3[MLP_H];                 // BF16-rounded, as FP32
    float b3;
    float pad[3];
};
static_assert(sizeof(MlpTcImage) % 16 == 0, "weight image is copied in 16-byte words");

// byte offset of element (r, k) in the no-swizzle K-major image of an R x K matrix
__host__ __device__ constexpr int umma_kmajor_off(int r, int k, int K) {
    return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

inline float bf16_round(float f) {
    const unsigned int u = (unsigned int)bf16_bits(f) << 16;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

// Fill the weight image (host) from the FP32 parameters: B[n][k] = W[n][k]
// (the MMA computes D = A B^T with both operands K-major).
inline void mlp_pack_tc(const float* P, MlpTcImage& M) {
    memset(&M, 0, sizeof M);
    for (int n = 0; n < MLP_H; ++n) {
        for (int k = 0; k < 16; ++k)
            M.w1[umma_kmajor_off(n, k, 16) / 2] = bf16_bits(k < MLP_IN ? P[OFF_W1 + n * MLP_IN + k] : 0.f);
        for (int k = 0; k < MLP_H; ++k)
            M.w2[umma_kmajor_off(n, k, MLP_H) / 2] = bf16_bits(P[OFF_W2 + n * MLP_H + k]);
        M.b1[n] = P[OFF_B1 + n];
        M.b2[n] = P[OFF_B2 + n];
        M.w3[n] = bf16_round(P[OFF_W3 + n]);
    }
    M.b3 = P[OFF_B3];
}

struct MlpTcSmem {
    alignas(128) unsigned short a1[2][128 * 16];  // layer 1 A operands (features), tiles 0 and 1
    alignas(128) unsigned short a2[2][128 * MLP_H];  // layer 2 A operands (tanh of layer 1)
    alignas(128) MlpTcImage W;
    unsigned long long bar;  // MMA completion
    unsigned int tmem;       // TMEM base address from tcgen05.alloc
};
constexpr int MLP_TC_COLS = 64;  // TMEM columns: tile 0 accumulators 0..31, tile 1 32..63
// With this footprint at most 8 CTAs fit on an SM (228 KB of shared memory,
// 1 KB reserved per CTA), so their 64-column TMEM allocations (8 x 64 = 512
// columns) never wait for one another.
static_assert(9 * (sizeof(MlpTcSmem) + 1024) > 228 * 1024, "TMEM columns would be oversubscribed");

// Shared-memory matrix descriptor: start address, leading (K) byte offset,
// stride (8-row group) byte offset, descriptor version 1, no swizzle.
__device__ __forceinline__ unsigned long long umma_desc(const void* p, unsigned lbo, unsigned sbo) {
    return (unsigned long long)((smem_u32(p) & 0x3FFFFu) >> 4) | ((unsigned long long)(lbo >> 4) << 16) |
           ((unsigned long long)(sbo >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 32, M = 128.
constexpr unsigned MLP_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(MLP_H >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(unsigned tmem_d, unsigned long long da, unsigned long long db, int acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(MLP_IDESC), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp-collective)
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// two FP32 values to packed BF16 (round to nearest even), lo in the low half
__device__ __forceinline__ unsigned int pack2_rn(float lo, float hi) {
    unsigned int r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// CTA set-up: weights into shared memory, the MMA barrier, and the TMEM
// columns (allocated by warp 0, which also frees them in mlp_tc_teardown).
__device__ __forceinline__ void mlp_tc_setup(MlpTcSmem& S, const MlpTcImage* __restrict__ Mg) {
    const uint4* src = reinterpret_cast<const uint4*>(Mg);
    uint4* dst = reinterpret_cast<uint4*>(&S.W);
    for (int k = threadIdx.x; k < (int)(sizeof(MlpTcImage) / 16); k += blockDim.x) dst[k] = src[k];
    if (threadIdx.x == 0) mbar_init(&S.bar);
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(MLP_TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ __forceinline__ void mlp_tc_teardown(MlpTcSmem& S) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(MLP_TC_COLS)
                     : "memory");
    }
}

// Write this thread's 6 features as row t of layer 1's A operand of tile j.
__device__ __forceinline__ void mlp_tc_put_features(MlpTcSmem& S, int j, const float (&f)[MLP_IN]) {
    const int t = threadIdx.x;
    uint4 lo, hi;
    lo.x = pack2_rn(f[0], f[1]);
    lo.y = pack2_rn(f[2], f[3]);
    lo.z = pack2_rn(f[4], f[5]);
    lo.w = 0u;
    hi.x = hi.y = hi.z = hi.w = 0u;
    unsigned char* base = reinterpret_cast<unsigned char*>(S.a1[j]);
    *reinterpret_cast<uint4*>(base + umma_kmajor_off(t, 0, 16)) = lo;
    *reinterpret_cast<uint4*>(base + umma_kmajor_off(t, 8, 16)) = hi;
}

// Wait for the phase `phase` of the MMA barrier (bounded); then TMEM reads may start.
__device__ __forceinline__ void mlp_tc_wait(MlpTcSmem& S, unsigned& phase, int* status) {
    if (!mbar_wait(&S.bar, phase & 1u) && status) atomicOr(status, 2);
    ++phase;
    tc_fence_after();
}

// The network for row t of both tiles (features already written with
// mlp_tc_put_features by every thread).  All 128 threads call this together;
// need0 / need1: this thread's row of tile 0 / 1 wants the output.  Rows are
// independent in the products, so a warp none of whose rows of a tile want
// it skips that tile's read-back and activations (its rows of the next
// operand keep stale values, whose results nobody reads); its output is 0.
__device__ __forceinline__ void mlp_tc_pair(MlpTcSmem& S, unsigned& phase, int* status, bool need0, bool need1,
                                            float& out0, float& out1) {
    const int t = threadIdx.x, w = t >> 5;
    const unsigned tm = S.tmem;
    const unsigned lane_base = (unsigned)(32 * w) << 16;
    const bool wj[2] = {__any_sync(0xffffffffu, need0) != 0, __any_sync(0xffffffffu, need1) != 0};
    // layer 1: D_j = A1_j W1^T
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
        tc_fence_after();
        const unsigned long long db = umma_desc(S.W.w1, 128, 16 * 16);
#pragma unroll
        for (int j = 0; j < 2; ++j) umma_bf16(tm + 32 * j, umma_desc(S.a1[j], 128, 16 * 16), db, 0);
        umma_commit(&S.bar);
    }
    mlp_tc_wait(S, phase, status);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        if (!wj[j]) continue;
        unsigned char* base = reinterpret_cast<unsigned char*>(S.a2[j]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float d[16];
            tmem_ld16(tm + lane_base + 32 * j + 16 * h, d);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int k0 = 16 * h + 8 * c;
                uint4 v;
                v.x = pack2_rn(tanh_fast(d[8 * c + 0] + S.W.b1[k0 + 0]), tanh_fast(d[8 * c + 1] + S.W.b1[k0 + 1]));
                v.y = pack2_rn(tanh_fast(d[8 * c + 2] + S.W.b1[k0 + 2]), tanh_fast(d[8 * c + 3] + S.W.b1[k0 + 3]));
                v.z = pack2_rn(tanh_fast(d[8 * c + 4] + S.W.b1[k0 + 4]), tanh_fast(d[8 * c + 5] + S.W.b1[k0 + 5]));
                v.w = pack2_rn(tanh_fast(d[8 * c + 6] + S.W.b1[k0 + 6]), tanh_fast(d[8 * c + 7] + S.W.b1[k0 + 7]));
                *reinterpret_cast<uint4*>(base + umma_kmajor_off(t, k0, MLP_H)) = v;
            }
        }
    }
    // layer 2: D_j = A2_j W2^T, two K = 16 steps (the K offset is two core matrices, 256 bytes)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
        tc_fence_after();
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int kk = 0; kk < 2; ++kk)
                umma_bf16(tm + 32 * j, umma_desc(reinterpret_cast<const unsigned char*>(S.a2[j]) + 256 * kk, 128, 16 * MLP_H),
                          umma_desc(reinterpret_cast<const unsigned char*>(S.W.w2) + 256 * kk, 128, 16 * MLP_H), kk);
        umma_commit(&S.bar);
    }
    mlp_tc_wait(S, phase, status);
    float o[2] = {0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        if (!wj[j]) continue;
        float acc = S.W.b3;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float d[16];
            tmem_ld16(tm + lane_base + 32 * j + 16 * h, d);
#pragma unroll
            for (int k = 0; k < 16; k += 2) {
                const unsigned int u =
                    pack2_rn(tanh_fast(d[k] + S.W.b2[16 * h + k]), tanh_fast(d[k + 1] + S.W.b2[16 * h + k + 1]));
                acc = fmaf(__uint_as_float(u << 16), S.W.w3[16 * h + k], acc);
                acc = fmaf(__uint_as_float(u & 0xffff0000u), S.W.w3[16 * h + k + 1], acc);
            }
        }
        o[j] = acc;
    }
    out0 = o[0];
    out1 = o[1];
    // the next pair's MMAs overwrite the accumulators and operands: every
    // thread's reads are done before any thread passes the next barrier
    tc_fence_before();
}

// Network outputs for n feature rows (x[i*8 + 0..5]) -- the raw evaluator
// behind claw2_mlp_infer: 256 rows per tile pair, CTAs loop over the pairs.
static __global__ void __launch_bounds__(128) k_mlp_eval_tc(const MlpTcImage* __restrict__ Mg,
                                                            const float* __restrict__ x, int n, float* y,
                                                            int* status) {
    __shared__ MlpTcSmem S;
    mlp_tc_setup(S, Mg);
    unsigned phase = 0;
    const int t = threadIdx.x;
    const int npairs = (n + 255) / 256;
    for (int pr = blockIdx.x; pr < npairs; pr += gridDim.x) {
        const long long r0 = (long long)pr * 256 + t, r1 = r0 + 128;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const long long r = j ? r1 : r0;
            float f[MLP_IN];
#pragma unroll
            for (int c = 0; c < MLP_IN; ++c) f[c] = (r < n) ? x[r * 8 + c] : 0.f;
            mlp_tc_put_features(S, j, f);
        }
        float o0, o1;
        mlp_tc_pair(S, phase, status, r0 < n, r1 < n, o0, o1);
        if (r0 < n) y[r0] = o0;
        if (r1 < n) y[r1] = o1;
    }
    mlp_tc_teardown(S);
}

// exact_euler::features in FP32 for the inference pass (the features enter
// the network as BF16, so FP32 arithmetic loses nothing that counts): a and
// b are the (rho, u, v, p, c) of the cells left/below and right/above, dir 1
// or 2 picks the normal velocity.  Non-finite features become 0; a
// non-finite jump weight leaves the interface to the PVRS guess.
__device__ __forceinline__ void features_f32(float g, const double (&a)[5], const double (&b)[5], int dir,
                                             float (&x)[MLP_IN], float& w) {
    const float rl = (float)a[0], ul = (float)a[dir], pl = (float)a[3];
    const float rr = (float)b[0], ur = (float)b[dir], pr = (float)b[3];
    const float rb = sqrtf(rl * rr), pb = sqrtf(pl * pr);
    const float cb = sqrtf(__fdividef(g * pb, rb));
    const float icb = __fdividef(1.f, cb);
    const float lr = 0.5f * __logf(__fdividef(rl, rr)), lp = 0.5f * __logf(__fdividef(pl, pr));
    x[0] = lr;
    x[1] = -lr;
    x[2] = ul * icb;
    x[3] = ur * icb;
    x[4] = lp;
    x[5] = -lp;
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) x[k] = isfinite(x[k]) ? x[k] : 0.f;
    const float dr = __fdividef(rr - rl, rb), dp = __fdividef(pr - pl, pb), du = (ur - ul) * icb;
    const float j2 = dr * dr + dp * dp + du * du;
    w = __fdividef(j2, 1.f + j2);
}

// Learned guesses for every interface of a grid (as k_mlp_guess, with the
// network on tcgen05): thread (cp, R) of a 32 x 4 site tile computes the
// x-interface (cp-1 | cp) on row R (tile 0, row t) and the y-interface
// (R-1 | R) on column cp (tile 1, row t).  CTAs loop over the site tiles.
static __global__ void __launch_bounds__(128, 5) k_mlp_guess_tc(const MlpTcImage* __restrict__ Mg,
                                                             const double* __restrict__ q, Layout L, double gamma,
                                                             double* guess, int* status) {
    __shared__ MlpTcSmem S;
    __shared__ double sprim[4][5][32];  // each warp's cells (rho, u, v, p, c): the row above's lower neighbours
    mlp_tc_setup(S, Mg);
    unsigned phase = 0;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tx = (L.mx + 4 + 31) / 32, ty = (L.my + 4 + 3) / 4;
    const long long ntiles = (long long)tx * ty;
    const exact_euler::Gas G = exact_euler::make_gas(gamma);
    const double g1 = gamma - 1.0;
    // primitive values and sound speed of one cell
    auto prim = [&](int cc, int rr, double (&v)[5]) {
        const long long o = (long long)rr * L.pitch + cc;
        const double rho = q[o], irho = rcp_nr(rho);
        v[0] = rho;
        v[1] = q[L.plane + o] * irho;
        v[2] = q[2 * L.plane + o] * irho;
        v[3] = g1 * (q[3 * L.plane + o] - 0.5 * rho * (v[1] * v[1] + v[2] * v[2]));
        v[4] = sqrt_nr(gamma * v[3] * irho);
    };
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int cp = (int)(tile % tx) * 32 + lane;
        const int R = (int)(tile / tx) * 4 + w;
        const int c = min(cp, L.mx + 3), r = min(R, L.my + 3);
        // this thread's cell; its left neighbour is the previous lane's cell
        // and its lower neighbour the previous warp's (each computed once),
        // except on the tile's first column and row
        double me[5], lf[5], lo[5];
        prim(c, r, me);
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            lf[k] = __shfl_up_sync(0xffffffffu, me[k], 1);
            sprim[w][k][lane] = me[k];
        }
        if (lane == 0) prim(max(c - 1, 0), r, lf);
        __syncthreads();
        if (w > 0) {
#pragma unroll
            for (int k = 0; k < 5; ++k) lo[k] = sprim[w - 1][k][lane];
        } else {
            prim(c, max(r - 1, 0), lo);
        }
        // features in FP32 (they enter the network as BF16)
        float wxf, wyf;
        float fx[MLP_IN], fy[MLP_IN];
        features_f32((float)gamma, lf, me, 1, fx, wxf);
        features_f32((float)gamma, lo, me, 2, fy, wyf);
        // PVRS decides: a weak jump (w below MLP_WMIN) keeps the PVRS guess;
        // a tile pair with only weak jumps skips the network
        const bool sx = wxf >= (float)MLP_WMIN, sy = wyf >= (float)MLP_WMIN;
        float ox = 0.f, oy = 0.f;
        if (__syncthreads_or(sx || sy)) {
            mlp_tc_put_features(S, 0, fx);
            mlp_tc_put_features(S, 1, fy);
            mlp_tc_pair(S, phase, status, sx, sy, ox, oy);
        }
        if (cp > L.mx + 3 || R > L.my + 3) continue;
        const double gx0 = exact_euler::guess_pvrs(G, lf[0], lf[1], lf[3], lf[4], me[0], me[1], me[3], me[4]);
        const double gy0 = exact_euler::guess_pvrs(G, lo[0], lo[2], lo[3], lo[4], me[0], me[2], me[3], me[4]);
        const long long o = (long long)R * L.pitch + cp;
        guess[o] = sx ? gx0 * (double)__expf(wxf * ox) : gx0;
        guess[L.plane + o] = sy ? gy0 * (double)__expf(wyf * oy) : gy0;
    }
    mlp_tc_teardown(S);
}

// The converged pressures as guesses (a measurement aid, no network): thread
// (cp, R) solves the x-interface (cp-1 | cp) and the y-interface (R-1 | R)
// exactly as the step kernel's Newton iteration would from the adaptive
// guess, to the same tolerance, and writes p* into the guess planes.  A step
// that starts from these needs no Newton update beyond the one that confirms
// convergence, so its time bounds from below what any guess can achieve.
// A deterministic number in [-1, 1) per interface (splitmix64 finaliser of
// its index): the sign and size of the error put on a converged guess.
__device__ __forceinline__ double guess_noise(unsigned long long k) {
    k += 0x9e3779b97f4a7c15ull;
    k = (k ^ (k >> 30)) * 0xbf58476d1ce4e5b9ull;
    k = (k ^ (k >> 27)) * 0x94d049bb133111ebull;
    k ^= k >> 31;
    return (double)(k >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// rel > 0: where the adaptive guess needs Newton steps, the converged p* is
// multiplied by 1 + rel * noise, noise in [-1, 1) -- a guess of that
// relative precision -- and elsewhere the step keeps the adaptive guess
// (guess 0): the most a guess of that precision can save with the adaptive
// guess as its fallback, used only where it would help.
static __global__ void __launch_bounds__(128) k_exact_pstar_guess(const double* __restrict__ q, Layout L,
                                                                  double gamma, double tol, double rel,
                                                                  double* guess) {
    const int cp = blockIdx.x * 32 + (threadIdx.x & 31);
    const int R = blockIdx.y * 4 + (threadIdx.x >> 5);
    if (cp > L.mx + 3 || R > L.my + 3) return;
    const exact_euler::Gas G = exact_euler::make_gas(gamma);
    const double g1 = gamma - 1.0;
    // the primitive values and sound speed exactly as RPEulerExact::prepare
    // forms them for the step, so the step's Newton starts at its own root
    auto prim = [&](int cc, int rr, double& rho, double& u, double& v, double& p, double& c) {
        const long long o = (long long)rr * L.pitch + cc;
        rho = q[o];
        const double irho = rcp_nr(rho);
        u = q[L.plane + o] * irho;
        v = q[2 * L.plane + o] * irho;
        p = g1 * (q[3 * L.plane + o] - 0.5 * (q[L.plane + o] * u + q[2 * L.plane + o] * v));
        c = sqrt_nr(gamma * p * irho);
    };
    double r0, u0, v0, p0, c0, rl, ul, vl, pl, cl, rb, ub, vb, pb, cb;
    prim(cp, R, r0, u0, v0, p0, c0);
    prim(max(cp - 1, 0), R, rl, ul, vl, pl, cl);
    prim(cp, max(R - 1, 0), rb, ub, vb, pb, cb);
    double ps, us;
    int it;
    const long long o = (long long)R * L.pitch + cp;
    guess[o] = 0.0;  // vacuum or a failed solve: the step falls back to the adaptive guess
    guess[L.plane + o] = 0.0;
    if (!exact_euler::vacuum(G, ul, cl, u0, c0)) {
        exact_euler::star(G, rl, ul, pl, cl, r0, u0, p0, c0, 0.0, tol, 50, ps, us, it);
        if (rel > 0.0) ps = it > 0 ? ps * (1.0 + rel * guess_noise(2ull * (unsigned long long)o)) : 0.0;
        guess[o] = ps;
    }
    if (!exact_euler::vacuum(G, vb, cb, v0, c0)) {
        exact_euler::star(G, rb, vb, pb, cb, r0, v0, p0, c0, 0.0, tol, 50, ps, us, it);
        if (rel > 0.0) ps = it > 0 ? ps * (1.0 + rel * guess_noise(2ull * (unsigned long long)o + 1ull)) : 0.0;
        guess[L.plane + o] = ps;
    }
}

}  // namespace claw2
