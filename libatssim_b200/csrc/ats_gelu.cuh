// ats_gelu.cuh -- the activation of the warm-start network.
//
// GELU in an FMA-only polynomial form:
//   g(z) = z (1/2 + z S(x)),  x = 2 z^2 / c^2 - 1,  |z| < c = 4.5;   g = z (z >= c), 0 (z <= -c)
// S is a degree-8 polynomial, the least-squares Chebyshev fit of (Phi(z) - 1/2) / z
// (Phi the standard normal CDF) weighted by z^2, in powers of x, generated by
// fit_gelu.py beside this file. g is within 1.2e-4 of z Phi(z) (the tanh form of GELU
// is within 4.8e-4) and jumps by 1.5e-5 at +-c; activations are rounded to BF16
// (2^-9 relative) right after it. It uses no transcendental-unit instruction, and the
// packed form evaluates two activations per FFMA2 (sm_100). The scalar and packed
// forms round identically (every step is one IEEE round-to-nearest operation), so
// training, inference and the CPU oracle evaluate the same function.
#pragma once

#include <cuda_runtime.h>

namespace ats {

constexpr float kGeluCut = 4.5f;
constexpr float kGeluScale = 0.0987654321f;  // 2 / c^2
constexpr int kGeluDeg = 8;
// S(x) = sum_k kGeluPoly[k] x^k, lowest power first
static __constant__ float kGeluPoly[kGeluDeg + 1] = {
    1.569028050e-01f, -7.717044652e-02f, 5.479086563e-02f, -4.057224095e-02f, 2.779665403e-02f,
    -1.670240983e-02f, 1.189577673e-02f, -9.356983006e-03f, 3.531820374e-03f};

__device__ __forceinline__ float gelu_tail(float z, float g) {
    return z >= kGeluCut ? z : (z <= -kGeluCut ? 0.f : g);
}

__device__ __forceinline__ float gelu(float z) {
    const float x = fmaf(__fmul_rn(z, z), kGeluScale, -1.f);
    float s = kGeluPoly[kGeluDeg];
#pragma unroll
    for (int k = kGeluDeg - 1; k >= 0; --k) s = fmaf(s, x, kGeluPoly[k]);
    return gelu_tail(z, __fmul_rn(z, fmaf(z, s, 0.5f)));
}

// two activations at once (FFMA2 / FMUL2), bitwise equal to gelu() on each
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 x = __ffma2_rn(__fmul2_rn(z, z), make_float2(kGeluScale, kGeluScale), make_float2(-1.f, -1.f));
    float2 s = make_float2(kGeluPoly[kGeluDeg], kGeluPoly[kGeluDeg]);
#pragma unroll
    for (int k = kGeluDeg - 1; k >= 0; --k) s = __ffma2_rn(s, x, make_float2(kGeluPoly[k], kGeluPoly[k]));
    const float2 g = __fmul2_rn(z, __ffma2_rn(z, s, make_float2(0.5f, 0.5f)));
    return make_float2(gelu_tail(z.x, g.x), gelu_tail(z.y, g.y));
}

// g'(z) = 1/2 + 2 z S(x) + 2 kGeluScale z^3 S'(x)
__device__ __forceinline__ float gelu_grad(float z) {
    const float x = fmaf(__fmul_rn(z, z), kGeluScale, -1.f);
    float s = kGeluPoly[kGeluDeg], d = 0.f;
#pragma unroll
    for (int k = kGeluDeg - 1; k >= 0; --k) {
        d = fmaf(d, x, s);
        s = fmaf(s, x, kGeluPoly[k]);
    }
    const float g = 0.5f + 2.f * z * s + 2.f * kGeluScale * z * z * z * d;
    return z >= kGeluCut ? 1.f : (z <= -kGeluCut ? 0.f : g);
}

}  // namespace ats
