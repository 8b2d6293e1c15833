// ats_learn.cu -- learned warm start for the VBD frame (no counterpart in the reference).
//
// A per-vertex MLP predicts the frame's solved position from local features; the
// plain VBD iterations always run afterwards. Per vertex v, with y the inertial
// prediction, h the substep and s = 9.8 h^2 (the gravity displacement of one step):
//   features (24): h v / s, (y - x0) / s, and for the 6 edge neighbours in rest
//   directions (+x, +x+z, +z, -x, -x-z, -z) (x0_u - x0_v) / rest length (0 if none)
//   output (3):    (x* - y) / s,   guess = y + s * output   (pinned vertices keep y)
// Network 24 -> 64 -> 64 -> 64 -> 3, GELU (polynomial form, ats_gelu.cuh), BF16 weights
// and activations, FP32 accumulation on the tensor cores: inference by tcgen05 MMA with
// TMEM accumulators (infer_tc_kernel), training by mma.sync m16n8k16 (train_tile_kernel).
// Training: MSE on the solved positions of recorded frames, Adam, deterministic per-CTA
// gradient partials.
// Fallback: per instance, the guess is kept only if the FP64 incremental potential
// G(guess) <= G(y) (Energy::compute_energy_* terms, xpbd_constraints.h:2079-2214).

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <memory>
#include <vector>

#include "ats_gelu.cuh"
#include "ats_internal.cuh"
#include "ats_umma.cuh"

namespace ats {
namespace {

constexpr int kIn = 24, kInP = 32, kHid = 64, kOut = 3, kOutP = 16;
constexpr int kTile = 64;      // samples per CTA
constexpr int kThreads = 128;  // 4 warps
// FP32 master parameter layout: W[in][out] row-major, then bias, per layer
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid * kHid, kW4 = kB3 + kHid, kB4 = kW4 + kHid * kOut, kParams = kB4 + kOut;
static_assert(kParams == 10115, "24-64-64-64-3 MLP has 10115 parameters");
// BF16 packed weights, transposed [out][in] with zero padding: W1t[64][32], W2t[64][64],
// W3t[64][64], W4t[16][64]
constexpr int kP1 = 0, kP2 = kP1 + kHid * kInP, kP3 = kP2 + kHid * kHid, kP4 = kP3 + kHid * kHid,
              kPacked = kP4 + kOutP * kHid;
// normalisation: in_mean[24], in_scale[24] (1/std), out_mean[3], out_std[3]; the network
// sees (f - in_mean) * in_scale and predicts (target - out_mean) / out_std
constexpr int kNormInMean = 0, kNormInScale = kIn, kNormOutMean = 2 * kIn, kNormOutStd = 2 * kIn + kOut,
              kNorm = 2 * kIn + 2 * kOut;

// ---------------------------------------------------------------- tensor-core tile GEMM
__device__ __forceinline__ uint32_t pk(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma16816(float d[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// C[M][N] = sum_k A(m, k) B(k, n) over the CTA's 4 warps, one 16x8 output tile per
// mma chain; A and B return BF16 elements (any layout), epi(m, n, value) consumes
// the FP32 result. Fragment layout of m16n8k16 (PTX ISA): group g = lane/4, thread
// t = lane%4; A rows g / g+8, columns 2t.. / 2t+8..; B columns g, rows 2t.. / 2t+8...
// The accumulators start at init(n) (a bias, or 0).
template <int M, int N, int K, typename FA, typename FB, typename FI, typename FE>
__device__ __forceinline__ void cta_gemm_init(FA A, FB B, FI init, FE epi) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    constexpr int MT = M / 16, NT = N / 8;
    for (int tile = warp; tile < MT * NT; tile += kThreads / 32) {
        const int m0 = (tile / NT) * 16, n0 = (tile % NT) * 8;
        const float i0 = init(n0 + 2 * t), i1 = init(n0 + 2 * t + 1);
        float d[4] = {i0, i1, i0, i1};
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 16) {
            const uint32_t a0 = pk(A(m0 + g, k0 + 2 * t), A(m0 + g, k0 + 2 * t + 1));
            const uint32_t a1 = pk(A(m0 + g + 8, k0 + 2 * t), A(m0 + g + 8, k0 + 2 * t + 1));
            const uint32_t a2 = pk(A(m0 + g, k0 + 2 * t + 8), A(m0 + g, k0 + 2 * t + 9));
            const uint32_t a3 = pk(A(m0 + g + 8, k0 + 2 * t + 8), A(m0 + g + 8, k0 + 2 * t + 9));
            const uint32_t b0 = pk(B(k0 + 2 * t, n0 + g), B(k0 + 2 * t + 1, n0 + g));
            const uint32_t b1 = pk(B(k0 + 2 * t + 8, n0 + g), B(k0 + 2 * t + 9, n0 + g));
            mma16816(d, a0, a1, a2, a3, b0, b1);
        }
        epi(m0 + g, n0 + 2 * t, d[0]);
        epi(m0 + g, n0 + 2 * t + 1, d[1]);
        epi(m0 + g + 8, n0 + 2 * t, d[2]);
        epi(m0 + g + 8, n0 + 2 * t + 1, d[3]);
    }
}

template <int M, int N, int K, typename FA, typename FB, typename FE>
__device__ __forceinline__ void cta_gemm(FA A, FB B, FE epi) {
    cta_gemm_init<M, N, K>(A, B, [](int) { return 0.f; }, epi);
}

// Shared memory of one 64-sample tile.
struct Tile {
    __nv_bfloat16 w[kPacked];        // packed weights
    float b[3 * kHid + kOutP];       // biases (b4 padded)
    __nv_bfloat16 x[kTile][kInP];    // features
    float z[3][kTile][kHid];         // pre-activations (with bias) of the hidden layers
    __nv_bfloat16 h[3][kTile][kHid]; // activations
    float y[kTile][kOutP];           // outputs
    __nv_bfloat16 dz[kTile][kHid];   // BF16 gradient of the current pre-activation
    __nv_bfloat16 dy[kTile][kOutP];
    float dzf[kTile][kHid];          // FP32 gradient (bias sums, GELU')
    float t[kTile][kOut];            // targets (normalised)
    float loss[kThreads];
    float nrm[kNorm];                // normalisation
};

__device__ void load_weights(Tile& S, const __nv_bfloat16* wpack, const float* master, const float* nrm) {
    for (int i = threadIdx.x; i < kNorm; i += kThreads) S.nrm[i] = nrm[i];
    for (int i = threadIdx.x; i < kPacked; i += kThreads) S.w[i] = wpack[i];
    for (int i = threadIdx.x; i < kHid; i += kThreads) {
        S.b[i] = master[kB1 + i];
        S.b[kHid + i] = master[kB2 + i];
        S.b[2 * kHid + i] = master[kB3 + i];
    }
    for (int i = threadIdx.x; i < kOutP; i += kThreads) S.b[3 * kHid + i] = i < kOut ? master[kB4 + i] : 0.f;
}

// Forward pass of the tile in shared memory (x filled, weights loaded).
__device__ void forward(Tile& S) {
    const __nv_bfloat16* W1 = S.w + kP1;
    const __nv_bfloat16* W2 = S.w + kP2;
    const __nv_bfloat16* W3 = S.w + kP3;
    const __nv_bfloat16* W4 = S.w + kP4;
    // the accumulators start at the bias: z = b + sum_k a_k w_k
    cta_gemm_init<kTile, kHid, kInP>([&](int m, int k) { return S.x[m][k]; },
                                     [&](int k, int n) { return W1[n * kInP + k]; }, [&](int n) { return S.b[n]; },
                                     [&](int m, int n, float v) {
                                         S.z[0][m][n] = v;
                                         S.h[0][m][n] = __float2bfloat16_rn(gelu(v));
                                     });
    __syncthreads();
    cta_gemm_init<kTile, kHid, kHid>([&](int m, int k) { return S.h[0][m][k]; },
                                     [&](int k, int n) { return W2[n * kHid + k]; },
                                     [&](int n) { return S.b[kHid + n]; },
                                     [&](int m, int n, float v) {
                                         S.z[1][m][n] = v;
                                         S.h[1][m][n] = __float2bfloat16_rn(gelu(v));
                                     });
    __syncthreads();
    cta_gemm_init<kTile, kHid, kHid>([&](int m, int k) { return S.h[1][m][k]; },
                                     [&](int k, int n) { return W3[n * kHid + k]; },
                                     [&](int n) { return S.b[2 * kHid + n]; },
                                     [&](int m, int n, float v) {
                                         S.z[2][m][n] = v;
                                         S.h[2][m][n] = __float2bfloat16_rn(gelu(v));
                                     });
    __syncthreads();
    cta_gemm_init<kTile, kOutP, kHid>([&](int m, int k) { return S.h[2][m][k]; },
                                      [&](int k, int n) { return W4[n * kHid + k]; },
                                      [&](int n) { return S.b[3 * kHid + n]; },
                                      [&](int m, int n, float v) { S.y[m][n] = v; });
    __syncthreads();
}

// Backward pass: gradient of sum over valid rows of (y - t)^2 * inv_count, written as
// FP32 partials grad[kParams] of this tile; returns nothing, loss in S.loss.
__device__ void backward(Tile& S, int valid, float inv_count, float* grad) {
    const __nv_bfloat16* W2 = S.w + kP2;
    const __nv_bfloat16* W3 = S.w + kP3;
    const __nv_bfloat16* W4 = S.w + kP4;
    // dL/dy = 2 (y - t) / count
    float lsum = 0.f;
    for (int i = threadIdx.x; i < kTile * kOutP; i += kThreads) {
        const int m = i / kOutP, n = i % kOutP;
        float g = 0.f;
        if (m < valid && n < kOut) {
            const float e = S.y[m][n] - S.t[m][n];
            lsum += e * e;
            g = 2.f * e * inv_count;
        }
        S.dzf[m][n] = g;  // FP32 copy for the bias (columns < kOutP)
        S.dy[m][n] = __float2bfloat16_rn(g);
    }
    S.loss[threadIdx.x] = lsum;
    __syncthreads();
    // layer 4: dW4[k][n] = sum_m h3[m][k] dy[m][n], db4 = sum_m dy
    cta_gemm<kHid, kOutP, kTile>([&](int k, int m) { return S.h[2][m][k]; }, [&](int m, int n) { return S.dy[m][n]; },
                                 [&](int k, int n, float v) {
                                     if (n < kOut) grad[kW4 + k * kOut + n] = v;
                                 });
    if (threadIdx.x < kOut) {
        float s = 0.f;
        for (int m = 0; m < kTile; ++m) s += S.dzf[m][threadIdx.x];
        grad[kB4 + threadIdx.x] = s;
    }
    __syncthreads();
    // dh3 = dy W4^T, dz3 = dh3 * gelu'(z3)
    cta_gemm<kTile, kHid, kOutP>([&](int m, int n) { return S.dy[m][n]; }, [&](int n, int k) { return W4[n * kHid + k]; },
                                 [&](int m, int k, float v) {
                                     const float g = v * gelu_grad(S.z[2][m][k]);
                                     S.dzf[m][k] = g;
                                     S.dz[m][k] = __float2bfloat16_rn(g);
                                 });
    __syncthreads();
    // hidden layers 3, 2 (weights W3, W2 and inputs h2, h1)
    for (int l = 2; l >= 1; --l) {
        const __nv_bfloat16* W = l == 2 ? W3 : W2;
        const int wofs = l == 2 ? kW3 : kW2, bofs = l == 2 ? kB3 : kB2;
        cta_gemm<kHid, kHid, kTile>([&](int k, int m) { return S.h[l - 1][m][k]; },
                                    [&](int m, int n) { return S.dz[m][n]; },
                                    [&](int k, int n, float v) { grad[wofs + k * kHid + n] = v; });
        for (int n = threadIdx.x; n < kHid; n += kThreads) {
            float s = 0.f;
            for (int m = 0; m < kTile; ++m) s += S.dzf[m][n];
            grad[bofs + n] = s;
        }
        __syncthreads();
        // dh_{l-1} = dz W^T ; dz_{l-1} = dh * gelu'(z_{l-1}); staged in y-sized scratch? use dzf
        cta_gemm<kTile, kHid, kHid>([&](int m, int n) { return S.dz[m][n]; }, [&](int n, int k) { return W[n * kHid + k]; },
                                    [&](int m, int k, float v) { S.z[l][m][k] = v * gelu_grad(S.z[l - 1][m][k]); });
        __syncthreads();
        for (int i = threadIdx.x; i < kTile * kHid; i += kThreads) {
            const int m = i / kHid, k = i % kHid;
            const float g = S.z[l][m][k];
            S.dzf[m][k] = g;
            S.dz[m][k] = __float2bfloat16_rn(g);
        }
        __syncthreads();
    }
    // layer 1: dW1[k][n] = sum_m x[m][k] dz1[m][n] (k < 24), db1
    cta_gemm<kInP, kHid, kTile>([&](int k, int m) { return S.x[m][k]; }, [&](int m, int n) { return S.dz[m][n]; },
                                [&](int k, int n, float v) {
                                    if (k < kIn) grad[kW1 + k * kHid + n] = v;
                                });
    for (int n = threadIdx.x; n < kHid; n += kThreads) {
        float s = 0.f;
        for (int m = 0; m < kTile; ++m) s += S.dzf[m][n];
        grad[kB1 + n] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// One training tile per CTA: samples are drawn uniformly from the dataset (seeded),
// or taken in order when `draw` is 0 (gradient check).
__global__ void __launch_bounds__(kThreads) train_tile_kernel(const float* __restrict__ feat, const float* __restrict__ targ,
                                                              long long n_data, int batch, int draw, uint64_t seed,
                                                              const __nv_bfloat16* wpack, const float* master,
                                                              const float* nrm, float* partial, float* loss_partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    Tile& S = *reinterpret_cast<Tile*>(smem);
    load_weights(S, wpack, master, nrm);
    __syncthreads();
    const int base = blockIdx.x * kTile;
    const int valid = max(0, min(kTile, batch - base));
    for (int i = threadIdx.x; i < kTile; i += kThreads) {
        long long idx = 0;
        const bool ok = i < valid;
        if (ok) idx = draw ? (long long)(mix64(seed ^ ((uint64_t)(base + i) * 0x632BE59BD9B4E019ull)) % (uint64_t)n_data)
                           : (long long)(base + i);
        for (int k = 0; k < kInP; ++k)
            S.x[i][k] = __float2bfloat16_rn(
                ok && k < kIn ? (feat[idx * kIn + k] - S.nrm[kNormInMean + k]) * S.nrm[kNormInScale + k] : 0.f);
        for (int k = 0; k < kOut; ++k)
            S.t[i][k] = ok ? (targ[idx * kOut + k] - S.nrm[kNormOutMean + k]) / S.nrm[kNormOutStd + k] : 0.f;
    }
    __syncthreads();
    forward(S);
    backward(S, valid, 1.f / (float)(batch * kOut), partial + (size_t)blockIdx.x * kParams);
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < kThreads; ++i) s += S.loss[i];
        loss_partial[blockIdx.x] = s;
    }
}

// Sums the CTA partials in order, then Adam on the FP32 master and the BF16 packing.
__global__ void reduce_adam_kernel(const float* partial, int nparts, float* master, float* m1, float* m2, float* grad_out,
                                   __nv_bfloat16* wpack, float lr, float b1, float b2, float eps, int step, int apply) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.f;
    for (int c = 0; c < nparts; ++c) g += partial[(size_t)c * kParams + p];
    if (grad_out) grad_out[p] = g;
    if (!apply) return;
    const float a = b1 * m1[p] + (1.f - b1) * g;
    const float b = b2 * m2[p] + (1.f - b2) * g * g;
    m1[p] = a;
    m2[p] = b;
    const float ah = a / (1.f - powf(b1, (float)step)), bh = b / (1.f - powf(b2, (float)step));
    const float w = master[p] - lr * ah / (sqrtf(bh) + eps);
    master[p] = w;
    // packed (transposed) BF16 location of parameter p
    int at = -1;
    if (p < kB1) at = kP1 + (p % kHid) * kInP + p / kHid;
    else if (p >= kW2 && p < kB2) at = kP2 + ((p - kW2) % kHid) * kHid + (p - kW2) / kHid;
    else if (p >= kW3 && p < kB3) at = kP3 + ((p - kW3) % kHid) * kHid + (p - kW3) / kHid;
    else if (p >= kW4 && p < kB4) at = kP4 + ((p - kW4) % kOut) * kHid + (p - kW4) / kOut;
    if (at >= 0) wpack[at] = __float2bfloat16_rn(w);
}

__global__ void sum_loss_kernel(const float* loss_partial, int n, float* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; ++i) s += loss_partial[i];
        *out = s;
    }
}

// Per-column sums of x and x^2 (FP64) of an n x cols array; block b takes rows
// b, b + gridDim.x, ... and writes its partials; one thread per column.
__global__ void column_moments_kernel(const float* __restrict__ a, long long n, int cols, double* partial) {
    const int c = threadIdx.x;
    if (c >= cols) return;
    double s = 0.0, s2 = 0.0;
    for (long long r = blockIdx.x; r < n; r += gridDim.x) {
        const double v = a[r * cols + c];
        s += v;
        s2 += v * v;
    }
    partial[(size_t)blockIdx.x * 2 * cols + c] = s;
    partial[(size_t)blockIdx.x * 2 * cols + cols + c] = s2;
}

// ---------------------------------------------------------------- features and inference
struct FeatArgs {
    const float4* x0;
    const float4* vel;
    const float4* vm;
    const float4* inst;
    const int* nb;      // 6 per vertex
    const float* len;   // 6 per vertex
    float h, inv_s;
    int nv;
};

__device__ __forceinline__ void vertex_features(const FeatArgs& a, int v, float f[kIn]) {
    const float4 p = a.x0[v], vv = a.vel[v], m = a.vm[v];
    const float4 acc = a.inst[__float_as_int(m.w)];
    const bool pinned = m.y != 0.f;
    const float hv[3] = {a.h * vv.x, a.h * vv.y, a.h * vv.z};
    const float ac[3] = {acc.x, acc.y, acc.z};
    for (int k = 0; k < 3; ++k) {
        f[k] = hv[k] * a.inv_s;
        f[3 + k] = pinned ? 0.f : (hv[k] + a.h * a.h * ac[k]) * a.inv_s;
    }
    for (int q = 0; q < 6; ++q) {
        const int u = a.nb[6 * v + q];
        if (u >= 0) {
            const float4 pu = a.x0[u];
            const float il = 1.f / a.len[6 * v + q];
            f[6 + 3 * q] = (pu.x - p.x) * il;
            f[7 + 3 * q] = (pu.y - p.y) * il;
            f[8 + 3 * q] = (pu.z - p.z) * il;
        } else {
            f[6 + 3 * q] = f[7 + 3 * q] = f[8 + 3 * q] = 0.f;
        }
    }
}

__global__ void features_kernel(FeatArgs a, float* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.nv) return;
    float f[kIn];
    vertex_features(a, v, f);
    for (int k = 0; k < kIn; ++k) out[(size_t)v * kIn + k] = f[k];
}

// Network outputs of n feature rows (the forward pass of ats_mlp_infer).
__global__ void __launch_bounds__(kThreads) infer_samples_kernel(const float* __restrict__ feat, int n,
                                                                 const __nv_bfloat16* wpack, const float* master,
                                                                 const float* nrm, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    Tile& S = *reinterpret_cast<Tile*>(smem);
    load_weights(S, wpack, master, nrm);
    __syncthreads();
    const int base = blockIdx.x * kTile;
    for (int i = threadIdx.x; i < kTile; i += kThreads) {
        const bool ok = base + i < n;
        for (int k = 0; k < kInP; ++k)
            S.x[i][k] = __float2bfloat16_rn(
                ok && k < kIn ? (feat[(size_t)(base + i) * kIn + k] - S.nrm[kNormInMean + k]) * S.nrm[kNormInScale + k]
                              : 0.f);
    }
    __syncthreads();
    forward(S);
    for (int i = threadIdx.x; i < kTile; i += kThreads)
        if (base + i < n)
            for (int k = 0; k < kOut; ++k)
                out[(size_t)(base + i) * kOut + k] = S.nrm[kNormOutMean + k] + S.nrm[kNormOutStd + k] * S.y[i][k];
}

__device__ __forceinline__ uint32_t pack_f2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// Inference on the 5th-generation tensor cores: one CTA of 128 threads per tile of 128
// vertices (the MMA's M), persistent over tiles. Thread r gathers vertex r's features
// into shared memory; one thread issues each layer as tcgen05.mma (BF16 operands from
// shared memory, FP32 accumulator in TMEM: layer 1 K = 32 as 2 steps of 16, the others
// K = 64 as 4); completion arrives on an mbarrier; every thread then reads its own row
// of the accumulator (tcgen05.ld, warp w owns TMEM lanes 32w..32w+31), adds the bias,
// applies the polynomial GELU in packed FP32 and writes the BF16 activations back as
// the next layer's A operand. TMEM columns: layers 1 and 3 at 0..63, 2 at 64..127, the
// output layer (N = 16, 3 used) at 64..79. Same quantisation points as the training
// forward (features and activations rounded to BF16, FP32 accumulation); the bias is
// added after the products instead of before, a different FP32 summation order.
constexpr int kTcRows = 128;
constexpr uint32_t kTcCols = 128;
constexpr uint32_t kTcWaitPolls = 1u << 24;
struct __align__(128) TcSmem {
    uint8_t w1[kHid * kInP * 2];      // W1^T, 64 x 32, K-major core matrices
    uint8_t w2[kHid * kHid * 2];      // W2^T, 64 x 64
    uint8_t w3[kHid * kHid * 2];      // W3^T
    uint8_t w4[kOutP * kHid * 2];     // W4^T, 16 x 64 (rows 3..15 zero)
    uint8_t a1[kTcRows * kInP * 2];   // features of the tile, 128 x 32
    uint8_t ah[kTcRows * kHid * 2];   // hidden activations, 128 x 64
    float b[3 * kHid + kOutP];
    float nrm[kNorm];
    uint64_t mbar;
    uint32_t tmem;
};
constexpr size_t kTcSmem = sizeof(TcSmem);
static_assert(offsetof(TcSmem, w2) % 128 == 0 && offsetof(TcSmem, w3) % 128 == 0 && offsetof(TcSmem, w4) % 128 == 0 &&
                  offsetof(TcSmem, a1) % 128 == 0 && offsetof(TcSmem, ah) % 128 == 0 && offsetof(TcSmem, mbar) % 8 == 0,
              "operand tiles 128-byte aligned");
static_assert(kTcSmem <= 56 * 1024, "at most 4 CTAs (4 x 128 TMEM columns) per SM");

// Rows of a packed [rows][K] BF16 matrix (global) into the K-major core-matrix layout.
__device__ __forceinline__ void tc_stage(uint8_t* dst, const __nv_bfloat16* src, int rows, int K) {
    const int chunks = rows * (K / 8);
    for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
        const int r = i / (K / 8), c = i % (K / 8);
        *reinterpret_cast<uint4*>(dst + umma::kmajor_offset(r, 8 * c, K)) =
            *reinterpret_cast<const uint4*>(src + (size_t)r * K + 8 * c);
    }
}

// One layer: D[tmem col dcol] = A (128 x K) * W^T (N x K)^T, issued by thread 0 after
// the CTA's shared-memory writes are visible to the tensor core; returns false (the
// same on every thread) if the completion wait ran out.
template <int K, int N>
__device__ __forceinline__ bool tc_layer(TcSmem& S, const uint8_t* a, const uint8_t* w, uint32_t dcol,
                                         uint32_t& phase) {
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        umma::fence_after_sync();
        constexpr uint32_t sbo = (K / 8) * 128;
        const uint32_t a0 = umma::smem_u32(a), w0 = umma::smem_u32(w);
#pragma unroll
        for (int s = 0; s < K / 16; ++s)
            umma::mma_bf16(S.tmem + dcol, umma::desc_kmajor(a0 + 256 * s, 128, sbo),
                           umma::desc_kmajor(w0 + 256 * s, 128, sbo), umma::idesc_bf16_f32(kTcRows, N), s > 0);
        umma::mma_commit(&S.mbar);
    }
    const bool ok = umma::mbar_wait(&S.mbar, phase, kTcWaitPolls);
    phase ^= 1u;
    umma::fence_after_sync();
    __syncwarp();
    return __syncthreads_and(ok) != 0;
}

// Row r of a hidden layer: TMEM (64 FP32) + bias -> GELU -> BF16 -> activation tile.
__device__ __forceinline__ void tc_hidden_epilogue(TcSmem& S, uint32_t dcol, const float* bias) {
    const int r = threadIdx.x;
    const uint32_t t = S.tmem + ((uint32_t)(r & ~31) << 16) + dcol;
    float lo[32], hi[32];
    umma::tmem_ld32(t, lo);
    umma::tmem_ld32(t + 32, hi);
    umma::tmem_ld_wait();
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        uint32_t q[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * c + 2 * j;
            const float z0 = (n < 32 ? lo[n] : hi[n - 32]) + bias[n];
            const float z1 = (n + 1 < 32 ? lo[n + 1] : hi[n + 1 - 32]) + bias[n + 1];
            const float2 g = gelu2(make_float2(z0, z1));
            q[j] = pack_f2(g.x, g.y);
        }
        *reinterpret_cast<uint4*>(S.ah + umma::kmajor_offset(r, 8 * c, kHid)) = make_uint4(q[0], q[1], q[2], q[3]);
    }
}

__global__ void __launch_bounds__(kTcRows, 1) infer_tc_kernel(FeatArgs fa, const __nv_bfloat16* __restrict__ wpack,
                                                              const float* __restrict__ master,
                                                              const float* __restrict__ nrm, float4* __restrict__ x,
                                                              float s, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t tc_smem_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_smem_raw);
    const int r = threadIdx.x, warp = r >> 5;
    tc_stage(S.w1, wpack + kP1, kHid, kInP);
    tc_stage(S.w2, wpack + kP2, kHid, kHid);
    tc_stage(S.w3, wpack + kP3, kHid, kHid);
    tc_stage(S.w4, wpack + kP4, kOutP, kHid);
    for (int i = r; i < kHid; i += kTcRows) {
        S.b[i] = master[kB1 + i];
        S.b[kHid + i] = master[kB2 + i];
        S.b[2 * kHid + i] = master[kB3 + i];
    }
    for (int i = r; i < kOutP; i += kTcRows) S.b[3 * kHid + i] = i < kOut ? master[kB4 + i] : 0.f;
    for (int i = r; i < kNorm; i += kTcRows) S.nrm[i] = nrm[i];
    if (warp == 0) umma::tmem_alloc(&S.tmem, kTcCols);
    if (r == 0) umma::mbar_init(&S.mbar, 1);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (fa.nv + kTcRows - 1) / kTcRows;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int v = tile * kTcRows + r;
        {
            float f[kIn];
            if (v < fa.nv) vertex_features(fa, v, f);
            uint32_t q[kInP / 2];
#pragma unroll
            for (int k = 0; k < kIn / 2; ++k)
                q[k] = v < fa.nv ? pack_f2((f[2 * k] - S.nrm[kNormInMean + 2 * k]) * S.nrm[kNormInScale + 2 * k],
                                           (f[2 * k + 1] - S.nrm[kNormInMean + 2 * k + 1]) *
                                               S.nrm[kNormInScale + 2 * k + 1])
                                 : 0u;
#pragma unroll
            for (int k = kIn / 2; k < kInP / 2; ++k) q[k] = 0u;
#pragma unroll
            for (int c = 0; c < kInP / 8; ++c)
                *reinterpret_cast<uint4*>(S.a1 + umma::kmajor_offset(r, 8 * c, kInP)) =
                    make_uint4(q[4 * c], q[4 * c + 1], q[4 * c + 2], q[4 * c + 3]);
        }
        if (!(ok = tc_layer<kInP, kHid>(S, S.a1, S.w1, 0, phase))) break;
        tc_hidden_epilogue(S, 0, S.b);
        if (!(ok = tc_layer<kHid, kHid>(S, S.ah, S.w2, 64, phase))) break;
        tc_hidden_epilogue(S, 64, S.b + kHid);
        if (!(ok = tc_layer<kHid, kHid>(S, S.ah, S.w3, 0, phase))) break;
        tc_hidden_epilogue(S, 0, S.b + 2 * kHid);
        if (!(ok = tc_layer<kHid, kOutP>(S, S.ah, S.w4, 64, phase))) break;
        float o[16];
        umma::tmem_ld16(S.tmem + ((uint32_t)(r & ~31) << 16) + 64, o);
        umma::tmem_ld_wait();
        if (v < fa.nv && fa.vm[v].y == 0.f) {
            float4 p = x[v];
            p.x += s * (S.nrm[kNormOutMean + 0] + S.nrm[kNormOutStd + 0] * (o[0] + S.b[3 * kHid + 0]));
            p.y += s * (S.nrm[kNormOutMean + 1] + S.nrm[kNormOutStd + 1] * (o[1] + S.b[3 * kHid + 1]));
            p.z += s * (S.nrm[kNormOutMean + 2] + S.nrm[kNormOutStd + 2] * (o[2] + S.b[3 * kHid + 2]));
            x[v] = p;
        }
    }
    if (!ok) {
        if (r == 0) atomicExch(err, 1);
        // an MMA may still be in flight: give it one more bounded wait before freeing TMEM
        umma::mbar_wait(&S.mbar, phase ^ 1u, kTcWaitPolls);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_free(S.tmem, kTcCols);
    }
}

__global__ void copy4_kernel(const float4* __restrict__ src, float4* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

// target = (x - y) / s of free vertices, appended in free-list order
__global__ void append_kernel(const float* __restrict__ stage, const float4* __restrict__ x, const float4* __restrict__ y,
                              const int* __restrict__ free_list, int nfree, float inv_s, float* __restrict__ feat,
                              float* __restrict__ targ, long long at) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfree) return;
    const int v = free_list[i];
    const size_t o = (size_t)(at + i);
    for (int k = 0; k < kIn; ++k) feat[o * kIn + k] = stage[(size_t)v * kIn + k];
    const float4 p = x[v], q = y[v];
    targ[o * kOut + 0] = (p.x - q.x) * inv_s;
    targ[o * kOut + 1] = (p.y - q.y) * inv_s;
    targ[o * kOut + 2] = (p.z - q.z) * inv_s;
}

// keep the guess of an instance only if G(guess) <= G(y); otherwise restore y
__global__ void fallback_kernel(float4* __restrict__ x, const float4* __restrict__ y, const float4* __restrict__ vm,
                                const double* gy, const double* gg, int* used, int nv, int ninst) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < ninst) used[v] = gg[v] <= gy[v] ? 1 : 0;
    if (v >= nv) return;
    const int i = __float_as_int(vm[v].w);
    if (!(gg[i] <= gy[i])) x[v] = y[v];
}

}  // namespace
}  // namespace ats

using namespace ats;

struct ats_mlp {
    DevBuf<float> master, m1, m2, grad, partial, loss_partial, loss, nrm;
    DevBuf<__nv_bfloat16> wpack;
    int step = 0;
    int partial_ctas = 0;
};

struct ats_dataset {
    DevBuf<float> feat, targ;
    long long capacity = 0, size = 0;
};

namespace {

constexpr size_t kTileSmem = sizeof(Tile);

int ensure_partials(ats_mlp* m, int ctas) {
    if (m->partial_ctas >= ctas) return ATS_OK;
    if (m->partial.p) {
        cudaFree(m->partial.p);
        m->partial.p = nullptr;
    }
    if (m->loss_partial.p) {
        cudaFree(m->loss_partial.p);
        m->loss_partial.p = nullptr;
    }
    ATS_CUDA(m->partial.alloc((size_t)ctas * kParams));
    ATS_CUDA(m->loss_partial.alloc(ctas));
    m->partial_ctas = ctas;
    return ATS_OK;
}

int g_tc_ctas = 148;     // CTAs of infer_tc_kernel: up to 4 per SM (shared memory, TMEM)

// Kernel attributes and launch shapes, set once before any launch or capture.
int set_smem_limits() {
    static bool done = false;
    if (done) return ATS_OK;
    {
        int dev = 0, sms = 0;
        ATS_CUDA(cudaGetDevice(&dev));
        ATS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        ATS_CUDA(cudaFuncSetAttribute(infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
        // the whole L1 / shared split as shared memory: four 48 KB CTAs per SM (with the
        // default split the runtime sized the SM for one)
        ATS_CUDA(cudaFuncSetAttribute(infer_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
        // 4 CTAs per SM: registers (119 x 128), shared memory (48 KB each) and TMEM
        // (4 x 128 of 512 columns) all admit four; the occupancy query reports one for
        // this kernel, and CTAs beyond what is resident simply start later (each works
        // alone on its tiles and frees its TMEM)
        int smem_optin = 0;
        ATS_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        const int by_smem = std::max(1, smem_optin / (int)(kTcSmem + 1024));
        const int tc_resident = std::min(by_smem, (int)(512 / kTcCols));
        g_tc_ctas = std::max(1, sms) * tc_resident;
    }
    ATS_CUDA(cudaFuncSetAttribute(train_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
    ATS_CUDA(cudaFuncSetAttribute(train_tile_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    ATS_CUDA(cudaFuncSetAttribute(infer_samples_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
    done = true;
    return ATS_OK;
}

void pack_host(const std::vector<float>& w, std::vector<__nv_bfloat16>& out) {
    out.assign(kPacked, __float2bfloat16(0.f));
    for (int k = 0; k < kIn; ++k)
        for (int n = 0; n < kHid; ++n) out[kP1 + n * kInP + k] = __float2bfloat16(w[kW1 + k * kHid + n]);
    for (int k = 0; k < kHid; ++k)
        for (int n = 0; n < kHid; ++n) {
            out[kP2 + n * kHid + k] = __float2bfloat16(w[kW2 + k * kHid + n]);
            out[kP3 + n * kHid + k] = __float2bfloat16(w[kW3 + k * kHid + n]);
        }
    for (int k = 0; k < kHid; ++k)
        for (int n = 0; n < kOut; ++n) out[kP4 + n * kHid + k] = __float2bfloat16(w[kW4 + k * kOut + n]);
}

int upload_params(ats_mlp* m, const std::vector<float>& w) {
    std::vector<__nv_bfloat16> pk;
    pack_host(w, pk);
    ATS_CUDA(cudaMemcpy(m->master.p, w.data(), kParams * sizeof(float), cudaMemcpyHostToDevice));
    ATS_CUDA(cudaMemcpy(m->wpack.p, pk.data(), kPacked * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
    ATS_CUDA(cudaMemset(m->m1.p, 0, kParams * sizeof(float)));
    ATS_CUDA(cudaMemset(m->m2.p, 0, kParams * sizeof(float)));
    m->step = 0;
    return ATS_OK;
}

FeatArgs feat_args(ats_cloth* c) {
    FeatArgs a;
    a.x0 = c->x0.p;
    a.vel = c->vel.p;
    a.vm = c->vm.p;
    a.inst = c->inst.p;
    a.nb = c->feat_nb.p;
    a.len = c->feat_len.p;
    a.h = c->h;
    a.inv_s = 1.f / (9.8f * c->h * c->h);
    a.nv = c->L.nv;
    return a;
}

int ensure_learn_buffers(ats_cloth* c) {
    const size_t nv = c->L.nv;
    if (!c->y_buf.p) ATS_CUDA(c->y_buf.alloc(nv));
    if (!c->pot_y.p) ATS_CUDA(c->pot_y.alloc(c->L.ninst));
    if (!c->pot_vx.p) ATS_CUDA(c->pot_vx.alloc(nv));  // per-vertex shares of G(guess), G(y)
    if (!c->pot_vy.p) ATS_CUDA(c->pot_vy.alloc(nv));
    if (!c->pot_guess.p) ATS_CUDA(c->pot_guess.alloc(c->L.ninst));
    if (!c->guess_used.p) ATS_CUDA(c->guess_used.alloc(c->L.ninst));
    if (!c->tc_err.p) {
        ATS_CUDA(c->tc_err.alloc(1));
        ATS_CUDA(cudaMemset(c->tc_err.p, 0, sizeof(int)));
    }
    return ATS_OK;
}

// The inference kernel's error flag, read (and cleared) after a synchronisation.
int check_tc_error(ats_cloth* c, cudaStream_t st) {
    if (!c->tc_err.p) return ATS_OK;
    int flag = 0;
    ATS_CUDA(cudaMemcpyAsync(&flag, c->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    if (!flag) return ATS_OK;
    ATS_CUDA(cudaMemsetAsync(c->tc_err.p, 0, sizeof(int), st));
    ATS_CUDA(cudaStreamSynchronize(st));
    set_error("warm-start inference: a tensor-core completion wait expired; the guess is incomplete");
    return ATS_ERR_TIMEOUT;
}

// after predict: save y, x = guess, then (G(guess), G(y) and the per-instance fallback)
int enqueue_warm_start(ats_cloth* c, const ats_mlp* m, int fallback, cudaStream_t st) {
    int r;
    if ((r = set_smem_limits()) || (r = ensure_learn_buffers(c))) return r;
    const int nv = c->L.nv;
    copy4_kernel<<<(nv + 255) / 256, 256, 0, st>>>(c->x.p, c->y_buf.p, nv); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    {
        const int tiles = (nv + kTcRows - 1) / kTcRows;
        const int grid = std::max(1, std::min(tiles, g_tc_ctas));
        infer_tc_kernel<<<grid, kTcRows, kTcSmem, st>>>(feat_args(c), m->wpack.p, m->master.p, m->nrm.p, c->x.p,
                                                        9.8f * c->h * c->h, c->tc_err.p); count_launch(st);
    }
    ATS_CUDA(cudaGetLastError());
    if (fallback) {
        if ((r = enqueue_potential_pair(c, c->y_buf.p, c->pot_guess.p, c->pot_y.p, st))) return r;
        const int n = std::max(nv, c->L.ninst);
        fallback_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->x.p, c->y_buf.p, c->vm.p, c->pot_y.p, c->pot_guess.p,
                                                          c->guess_used.p, nv, c->L.ninst); count_launch(st);
        ATS_CUDA(cudaGetLastError());
    }
    return ATS_OK;
}

std::vector<float> init_params(uint64_t seed) {
    std::vector<float> w(kParams, 0.f);
    uint64_t s = seed;
    auto next = [&]() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
    };
    auto fill = [&](int w0, int b0, int fan_in, int fan_out, float gain) {
        const float bound = gain / std::sqrt((float)fan_in);
        for (int i = 0; i < fan_in * fan_out; ++i) w[w0 + i] = (float)((2.0 * next() - 1.0) * bound);
        for (int i = 0; i < fan_out; ++i) w[b0 + i] = (float)((2.0 * next() - 1.0) * bound);
    };
    fill(kW1, kB1, kIn, kHid, 1.f);
    fill(kW2, kB2, kHid, kHid, 1.f);
    fill(kW3, kB3, kHid, kHid, 1.f);
    fill(kW4, kB4, kHid, kOut, 0.1f);  // small last layer: the first guesses stay close to y
    return w;
}

}  // namespace

extern "C" {

int ats_mlp_param_count(void) { return kParams; }

int ats_mlp_create(unsigned long long seed, ats_mlp** out) {
    if (!out) {
        set_error("ats_mlp_create: null output");
        return ATS_ERR_INVALID;
    }
    std::unique_ptr<ats_mlp> m(new (std::nothrow) ats_mlp());
    if (!m) {
        set_error("ats_mlp_create: out of memory");
        return ATS_ERR_NOMEM;
    }
    ATS_CUDA(m->master.alloc(kParams));
    ATS_CUDA(m->m1.alloc(kParams));
    ATS_CUDA(m->m2.alloc(kParams));
    ATS_CUDA(m->grad.alloc(kParams));
    ATS_CUDA(m->loss.alloc(1));
    ATS_CUDA(m->wpack.alloc(kPacked));
    ATS_CUDA(m->nrm.alloc(kNorm));
    {
        std::vector<float> id(kNorm, 0.f);
        for (int k = 0; k < kIn; ++k) id[kNormInScale + k] = 1.f;
        for (int k = 0; k < kOut; ++k) id[kNormOutStd + k] = 1.f;
        ATS_CUDA(cudaMemcpy(m->nrm.p, id.data(), kNorm * sizeof(float), cudaMemcpyHostToDevice));
    }
    int r = upload_params(m.get(), init_params(seed));
    if (r) return r;
    *out = m.release();
    return ATS_OK;
}

int ats_mlp_destroy(ats_mlp* m) {
    if (!m) return ATS_OK;
    cudaDeviceSynchronize();
    delete m;
    return ATS_OK;
}

int ats_mlp_get_params(const ats_mlp* m, float* out) {
    if (!m || !out) {
        set_error("ats_mlp_get_params: null argument");
        return ATS_ERR_INVALID;
    }
    ATS_CUDA(cudaMemcpy(out, m->master.p, kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return ATS_OK;
}

int ats_mlp_set_params(ats_mlp* m, const float* in) {
    if (!m || !in) {
        set_error("ats_mlp_set_params: null argument");
        return ATS_ERR_INVALID;
    }
    return upload_params(m, std::vector<float>(in, in + kParams));
}

int ats_mlp_get_normalization(const ats_mlp* m, float* norm) {
    if (!m || !norm) {
        set_error("ats_mlp_get_normalization: null argument");
        return ATS_ERR_INVALID;
    }
    ATS_CUDA(cudaMemcpy(norm, m->nrm.p, kNorm * sizeof(float), cudaMemcpyDeviceToHost));
    return ATS_OK;
}

int ats_mlp_set_normalization(ats_mlp* m, const float* norm) {
    if (!m || !norm) {
        set_error("ats_mlp_set_normalization: null argument");
        return ATS_ERR_INVALID;
    }
    for (int k = 0; k < kIn; ++k)
        if (!(norm[kNormInScale + k] > 0.f)) {
            set_error("ats_mlp_set_normalization: input scales must be > 0");
            return ATS_ERR_INVALID;
        }
    for (int k = 0; k < kOut; ++k)
        if (!(norm[kNormOutStd + k] > 0.f)) {
            set_error("ats_mlp_set_normalization: output std must be > 0");
            return ATS_ERR_INVALID;
        }
    ATS_CUDA(cudaMemcpy(m->nrm.p, norm, kNorm * sizeof(float), cudaMemcpyHostToDevice));
    return ATS_OK;
}

int ats_mlp_fit_normalization(ats_mlp* m, const ats_dataset* d, ats_stream stream) {
    if (!m || !d || d->size <= 1) {
        set_error("ats_mlp_fit_normalization: need a model and a dataset with at least 2 samples");
        return ATS_ERR_INVALID;
    }
    const int blocks = 256;
    DevBuf<double> pf, pt;
    ATS_CUDA(pf.alloc((size_t)blocks * 2 * kIn));
    ATS_CUDA(pt.alloc((size_t)blocks * 2 * kOut));
    cudaStream_t st = S(stream);
    column_moments_kernel<<<blocks, 32, 0, st>>>(d->feat.p, d->size, kIn, pf.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    column_moments_kernel<<<blocks, 32, 0, st>>>(d->targ.p, d->size, kOut, pt.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    std::vector<double> hf((size_t)blocks * 2 * kIn), ht((size_t)blocks * 2 * kOut);
    ATS_CUDA(cudaMemcpyAsync(hf.data(), pf.p, hf.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaMemcpyAsync(ht.data(), pt.p, ht.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    std::vector<float> nrm(kNorm);
    const double n = (double)d->size;
    auto stats = [&](const std::vector<double>& h, int cols, int c, double& mean, double& sd) {
        double s = 0.0, s2 = 0.0;
        for (int b = 0; b < blocks; ++b) {
            s += h[(size_t)b * 2 * cols + c];
            s2 += h[(size_t)b * 2 * cols + cols + c];
        }
        mean = s / n;
        sd = std::sqrt(std::max(s2 / n - mean * mean, 0.0));
        if (sd < 1e-6) sd = 1.0;  // a constant column (e.g. a zero-padded slot) is left unscaled
    };
    for (int k = 0; k < kIn; ++k) {
        double mu, sd;
        stats(hf, kIn, k, mu, sd);
        nrm[kNormInMean + k] = (float)mu;
        nrm[kNormInScale + k] = (float)(1.0 / sd);
    }
    for (int k = 0; k < kOut; ++k) {
        double mu, sd;
        stats(ht, kOut, k, mu, sd);
        nrm[kNormOutMean + k] = (float)mu;
        nrm[kNormOutStd + k] = (float)sd;
    }
    ATS_CUDA(cudaMemcpy(m->nrm.p, nrm.data(), kNorm * sizeof(float), cudaMemcpyHostToDevice));
    return ATS_OK;
}

int ats_dataset_create(long long capacity, ats_dataset** out) {
    if (!out || capacity <= 0) {
        set_error("ats_dataset_create: need capacity > 0 and an output pointer");
        return ATS_ERR_INVALID;
    }
    std::unique_ptr<ats_dataset> d(new (std::nothrow) ats_dataset());
    if (!d) {
        set_error("ats_dataset_create: out of memory");
        return ATS_ERR_NOMEM;
    }
    ATS_CUDA(d->feat.alloc((size_t)capacity * kIn));
    ATS_CUDA(d->targ.alloc((size_t)capacity * kOut));
    d->capacity = capacity;
    *out = d.release();
    return ATS_OK;
}

int ats_dataset_destroy(ats_dataset* d) {
    if (!d) return ATS_OK;
    cudaDeviceSynchronize();
    delete d;
    return ATS_OK;
}

int ats_dataset_size(const ats_dataset* d, long long* n) {
    if (!d || !n) {
        set_error("ats_dataset_size: null argument");
        return ATS_ERR_INVALID;
    }
    *n = d->size;
    return ATS_OK;
}

int ats_dataset_read(const ats_dataset* d, long long first, long long count, float* features, float* targets) {
    if (!d || first < 0 || count < 0 || first + count > d->size) {
        set_error("ats_dataset_read: range outside the dataset");
        return ATS_ERR_INVALID;
    }
    if (features)
        ATS_CUDA(cudaMemcpy(features, d->feat.p + first * kIn, count * kIn * sizeof(float), cudaMemcpyDeviceToHost));
    if (targets)
        ATS_CUDA(cudaMemcpy(targets, d->targ.p + first * kOut, count * kOut * sizeof(float), cudaMemcpyDeviceToHost));
    return ATS_OK;
}

int ats_record_frame_begin(ats_cloth* c, ats_stream stream) {
    if (!c) {
        set_error("ats_record_frame_begin: null handle");
        return ATS_ERR_INVALID;
    }
    int r = ensure_learn_buffers(c);
    if (r) return r;
    const int nv = c->L.nv;
    if (!c->feat_stage.p) ATS_CUDA(c->feat_stage.alloc((size_t)nv * kIn));
    if (!c->free_list.p) {
        std::vector<int> fl;
        for (int v = 0; v < nv; ++v)
            if (c->L.vm[4 * (size_t)v + 1] == 0.f) fl.push_back(v);
        ATS_CUDA(c->free_list.alloc(std::max<size_t>(1, fl.size())));
        c->free_list.n = fl.size();
        if (!fl.empty()) ATS_CUDA(cudaMemcpy(c->free_list.p, fl.data(), fl.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    cudaStream_t st = S(stream);
    copy4_kernel<<<(nv + 255) / 256, 256, 0, st>>>(c->x.p, c->y_buf.p, nv); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    features_kernel<<<(nv + 255) / 256, 256, 0, st>>>(feat_args(c), c->feat_stage.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    return ATS_OK;
}

int ats_record_frame_end(ats_cloth* c, ats_dataset* d, ats_stream stream) {
    if (!c || !d || !c->feat_stage.p) {
        set_error("ats_record_frame_end: need a handle with ats_record_frame_begin called, and a dataset");
        return ATS_ERR_INVALID;
    }
    const int nfree = (int)c->free_list.n;
    if (d->size + nfree > d->capacity) {
        set_error("ats_record_frame_end: dataset is full");
        return ATS_ERR_INVALID;
    }
    if (nfree > 0) {
        append_kernel<<<(nfree + 255) / 256, 256, 0, S(stream)>>>(c->feat_stage.p, c->x.p, c->y_buf.p, c->free_list.p, nfree,
                                                                  1.f / (9.8f * c->h * c->h), d->feat.p, d->targ.p, d->size); count_launch(S(stream));
        ATS_CUDA(cudaGetLastError());
    }
    d->size += nfree;
    return ATS_OK;
}

int ats_mlp_train(ats_mlp* m, const ats_dataset* d, int steps, int batch, float lr, unsigned long long seed,
                  float* mean_loss, ats_stream stream) {
    if (!m || !d || steps < 0 || batch <= 0 || d->size <= 0) {
        set_error("ats_mlp_train: need a model, a non-empty dataset, steps >= 0, batch > 0");
        return ATS_ERR_INVALID;
    }
    int r;
    const int ctas = (batch + kTile - 1) / kTile;
    if ((r = set_smem_limits()) || (r = ensure_partials(m, ctas))) return r;
    cudaStream_t st = S(stream);
    double loss_acc = 0.0;
    int loss_n = 0;
    for (int s = 0; s < steps; ++s) {
        ++m->step;
        train_tile_kernel<<<ctas, kThreads, kTileSmem, st>>>(d->feat.p, d->targ.p, d->size, batch, 1,
                                                              seed * 0x9E3779B97F4A7C15ull + (uint64_t)m->step,
                                                              m->wpack.p, m->master.p, m->nrm.p, m->partial.p,
                                                              m->loss_partial.p); count_launch(st);
        ATS_CUDA(cudaGetLastError());
        reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(m->partial.p, ctas, m->master.p, m->m1.p, m->m2.p,
                                                                  nullptr, m->wpack.p, lr, 0.9f, 0.999f, 1e-8f, m->step, 1); count_launch(st);
        ATS_CUDA(cudaGetLastError());
        if (mean_loss && s >= steps - std::min(steps, 20)) {
            float l = 0.f;
            sum_loss_kernel<<<1, 32, 0, st>>>(m->loss_partial.p, ctas, m->loss.p); count_launch(st);
            ATS_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
            ATS_CUDA(cudaStreamSynchronize(st));
            loss_acc += l / (double)(batch * kOut);
            ++loss_n;
        }
    }
    if (mean_loss) *mean_loss = loss_n ? (float)(loss_acc / loss_n) : 0.f;
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_mlp_batch_gradient(ats_mlp* m, const ats_dataset* d, int batch, unsigned long long seed, float* grad,
                           float* loss, ats_stream stream) {
    if (!m || !d || batch <= 0 || d->size <= 0 || !grad) {
        set_error("ats_mlp_batch_gradient: need a model, a non-empty dataset, batch > 0 and a gradient output");
        return ATS_ERR_INVALID;
    }
    int r;
    const int ctas = (batch + kTile - 1) / kTile;
    if ((r = set_smem_limits()) || (r = ensure_partials(m, ctas))) return r;
    cudaStream_t st = S(stream);
    train_tile_kernel<<<ctas, kThreads, kTileSmem, st>>>(d->feat.p, d->targ.p, d->size, batch, 1,
                                                          seed * 0x9E3779B97F4A7C15ull + 0x5851F42D4C957F2Dull,
                                                          m->wpack.p, m->master.p, m->nrm.p, m->partial.p,
                                                          m->loss_partial.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(m->partial.p, ctas, m->master.p, m->m1.p, m->m2.p,
                                                              m->grad.p, m->wpack.p, 0.f, 0.9f, 0.999f, 1e-8f, 1, 0); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    sum_loss_kernel<<<1, 32, 0, st>>>(m->loss_partial.p, ctas, m->loss.p); count_launch(st);
    ATS_CUDA(cudaMemcpyAsync(grad, m->grad.p, kParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    float l = 0.f;
    ATS_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    if (loss) *loss = l / (float)(batch * kOut);
    return ATS_OK;
}

int ats_mlp_apply_gradient(ats_mlp* m, const float* grad, float lr, ats_stream stream) {
    if (!m || !grad) {
        set_error("ats_mlp_apply_gradient: need a model and a gradient");
        return ATS_ERR_INVALID;
    }
    int r = ensure_partials(m, 1);
    if (r) return r;
    cudaStream_t st = S(stream);
    ATS_CUDA(cudaMemcpyAsync(m->partial.p, grad, kParams * sizeof(float), cudaMemcpyHostToDevice, st));
    ++m->step;
    reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(m->partial.p, 1, m->master.p, m->m1.p, m->m2.p, nullptr,
                                                              m->wpack.p, lr, 0.9f, 0.999f, 1e-8f, m->step, 1); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_mlp_gradient(ats_mlp* m, const float* features, const float* targets, int n, float* grad, float* loss,
                     ats_stream stream) {
    if (!m || !features || !targets || n <= 0 || !grad) {
        set_error("ats_mlp_gradient: need a model, n > 0 samples and a gradient output");
        return ATS_ERR_INVALID;
    }
    int r;
    const int ctas = (n + kTile - 1) / kTile;
    if ((r = set_smem_limits()) || (r = ensure_partials(m, ctas))) return r;
    DevBuf<float> f, t;
    ATS_CUDA(f.alloc((size_t)n * kIn));
    ATS_CUDA(t.alloc((size_t)n * kOut));
    cudaStream_t st = S(stream);
    ATS_CUDA(cudaMemcpyAsync(f.p, features, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice, st));
    ATS_CUDA(cudaMemcpyAsync(t.p, targets, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice, st));
    train_tile_kernel<<<ctas, kThreads, kTileSmem, st>>>(f.p, t.p, n, n, 0, 0, m->wpack.p, m->master.p, m->nrm.p,
                                                          m->partial.p, m->loss_partial.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(m->partial.p, ctas, m->master.p, m->m1.p, m->m2.p,
                                                              m->grad.p, m->wpack.p, 0.f, 0.9f, 0.999f, 1e-8f, 1, 0); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    sum_loss_kernel<<<1, 32, 0, st>>>(m->loss_partial.p, ctas, m->loss.p); count_launch(st);
    ATS_CUDA(cudaMemcpyAsync(grad, m->grad.p, kParams * sizeof(float), cudaMemcpyDeviceToHost, st));
    float l = 0.f;
    ATS_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    if (loss) *loss = l / (float)(n * kOut);
    return ATS_OK;
}

int ats_warm_start(ats_cloth* c, const ats_mlp* m, int fallback, int* used, ats_stream stream) {
    if (!c || !m) {
        set_error("ats_warm_start: need a handle and a model");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = enqueue_warm_start(c, m, fallback, st);
    if (r) return r;
    if (used) {
        if (fallback) {
            ATS_CUDA(cudaMemcpyAsync(used, c->guess_used.p, c->L.ninst * sizeof(int), cudaMemcpyDeviceToHost, st));
        } else {
            for (int i = 0; i < c->L.ninst; ++i) used[i] = 1;
        }
        ATS_CUDA(cudaStreamSynchronize(st));
        return check_tc_error(c, st);
    }
    return ATS_OK;
}

int ats_frame_warm(ats_cloth* c, const ats_mlp* m, int fallback, int iterations, int use_graph, ats_stream stream) {
    if (!c || !m) {
        set_error("ats_frame_warm: need a handle and a model");
        return ATS_ERR_INVALID;
    }
    const int iters = iterations < 0 ? c->prm.iterations : iterations;
    auto enqueue = [&](cudaStream_t st) {
        int r;
        for (int sub = 0; sub < c->prm.num_substep; ++sub) {
            if ((r = launch_predict(c, st)) || (r = enqueue_warm_start(c, m, fallback, st)) ||
                (r = enqueue_iterations(c, ATS_SOLVER_VBD, iters, st)) || (r = launch_update(c, st)))
                return r;
        }
        return (int)ATS_OK;
    };
    if (!use_graph) return enqueue(S(stream));
    int r;
    if ((r = set_smem_limits()) || (r = ensure_learn_buffers(c))) return r;
    // one captured warm frame per handle, re-captured when model, budget or fallback change
    if (!c->warm_graph || c->warm_key_mlp != (const void*)m || c->warm_key_iters != iters ||
        c->warm_key_fallback != fallback) {
        if (c->warm_graph) {
            cudaGraphExecDestroy(c->warm_graph);
            c->warm_graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        ATS_CUDA(cudaStreamBeginCapture(c->capture_stream, cudaStreamCaptureModeThreadLocal));
        r = enqueue(c->capture_stream);
        cudaError_t e = cudaStreamEndCapture(c->capture_stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) {
            set_error(std::string("ats_frame_warm: capture failed: ") + cudaGetErrorString(e));
            return ATS_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&c->warm_graph, g, 0);
        if (e == cudaSuccess) register_graph(c->warm_graph, g);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error(std::string("ats_frame_warm: instantiate failed: ") + cudaGetErrorString(e));
            return ATS_ERR_CUDA;
        }
        c->warm_key_mlp = m;
        c->warm_key_iters = iters;
        c->warm_key_fallback = fallback;
    }
    ATS_CUDA(cudaGraphLaunch(c->warm_graph, S(stream)));
    count_graph_launch(c->warm_graph);
    return ATS_OK;
}

int ats_frame_warm_to_residual(ats_cloth* c, const ats_mlp* m, int fallback, double tol, const double* tols,
                               const int* first_check, int check_every, int max_iterations, int* iterations,
                               double* residual, int* used, ats_stream stream) {
    if (!c || !m) {
        set_error("ats_frame_warm_to_residual: need a handle and a model");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = frame_to_residual_impl(c, tol, tols, first_check, check_every, max_iterations, iterations, residual, st,
                                   [&](cudaStream_t s) { return enqueue_warm_start(c, m, fallback, s); });
    if (r || (r = check_tc_error(c, st))) return r;
    if (used) {
        if (fallback) {
            ATS_CUDA(cudaMemcpyAsync(used, c->guess_used.p, c->L.ninst * sizeof(int), cudaMemcpyDeviceToHost, st));
            ATS_CUDA(cudaStreamSynchronize(st));
        } else {
            for (int i = 0; i < c->L.ninst; ++i) used[i] = 1;
        }
    }
    return ATS_OK;
}

int ats_mlp_infer(const ats_mlp* m, const float* features, int n, float* outputs, ats_stream stream) {
    if (!m || !features || !outputs || n <= 0) {
        set_error("ats_mlp_infer: need a model, n > 0 samples and an output array");
        return ATS_ERR_INVALID;
    }
    int r = set_smem_limits();
    if (r) return r;
    DevBuf<float> f, o;
    ATS_CUDA(f.alloc((size_t)n * kIn));
    ATS_CUDA(o.alloc((size_t)n * kOut));
    cudaStream_t st = S(stream);
    ATS_CUDA(cudaMemcpyAsync(f.p, features, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice, st));
    infer_samples_kernel<<<(n + kTile - 1) / kTile, kThreads, kTileSmem, st>>>(f.p, n, m->wpack.p, m->master.p,
                                                                                m->nrm.p, o.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaMemcpyAsync(outputs, o.p, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

}  // extern "C"
