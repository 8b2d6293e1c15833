// ats_kernels.cuh -- sm_100a kernels of the cloth solver.
//
// Data layout in HBM (all float4 = 16 B, one 128-bit load per vertex record):
//   x   [V]  current iterate, w unused
//   x0  [V]  frame / substep start position, w = mass
//   vel [V]  velocity, w = instance id (int bits)
//   vm  [V]  {k_b * sum Q_oo (bending Hessian diagonal), pin boost (0 / 1e9), inverse mass, k_stretch}
// Vertices are ordered instance-major then colour-major, so the vertices of one
// colour of one instance are contiguous and every own-vertex access of a sweep is
// coalesced. The neighbour stencil of a vertex (1-ring plus the far corners of its
// bending edges) is stored sliced-ELL: a slice is one warp, 32/TPV vertices with
// TPV lanes each; row r of a slice is 32 consecutive entries, entry (r, lane) is
// slot r*TPV + lane%TPV of vertex lane/TPV. Each row is one coalesced 128 B load
// per array (index, rest length, bending weight).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ats {

constexpr float kEps = 1.19209290E-7f;  // src/SharedDefine/constant_value.h:9

struct SweepArgs {
    float4* __restrict__ x;
    const float4* __restrict__ x0;
    const float4* __restrict__ vel;
    const float4* __restrict__ vm;
    const int* __restrict__ st_idx;
    const float* __restrict__ st_rest;
    const float* __restrict__ st_w;
    const int4* __restrict__ slices;
    const float4* __restrict__ accel;  // per instance, xyz
    int slice_begin, slice_end;
    float h, h2inv;
};

// One VBD colour sweep: for every vertex of the colour, inertia + mass-spring
// stretch + quadratic bending gradient and Hessian (reference:
// VBD::compute_inertia / compute_stretch_mass_spring / compute_bending_quadratic,
// xpbd_constraints.h:4027-4205), then the determinant-guarded 3x3 solve of
// example2_async_iter.cpp:993-1014, all in registers (Hf never goes to memory).
// Bending is linear in x, so the per-bending-edge terms -k_b sum_j Q[o][j] x_j are
// merged per (vertex, neighbour) into one weight W and applied in relative
// coordinates -sum_u W_vu (x_u - x_v), which is the same force because every row of
// Q sums to zero.
template <int TPV>
__global__ void __launch_bounds__(256) vbd_sweep_kernel(SweepArgs a) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int slice = a.slice_begin + warp;
    if (slice >= a.slice_end) return;
    const int lane = threadIdx.x & 31;
    const int4 sd = __ldg(&a.slices[slice]);  // vbegin, nverts, entry offset, rows
    const int k = lane / TPV;
    const bool active = k < sd.y;
    const int v = sd.x + min(k, sd.y - 1);
    const float4 xv = a.x[v];
    const float4 mv = __ldg(&a.vm[v]);
    const float ks = mv.w;

    float fx = 0.f, fy = 0.f, fz = 0.f;
    float h00 = 0.f, h01 = 0.f, h02 = 0.f, h11 = 0.f, h12 = 0.f, h22 = 0.f;
    const int base = sd.z + lane;
#pragma unroll 4
    for (int row = 0; row < sd.w; ++row) {
        const int e = base + row * 32;
        const int u = __ldg(&a.st_idx[e]);
        const float L = __ldg(&a.st_rest[e]);
        const float w = __ldg(&a.st_w[e]);
        // neighbours belong to other colours: nothing in this launch writes them
        const float4 xu = __ldg(&a.x[u]);
        const float dx = xu.x - xv.x, dy = xu.y - xv.y, dz = xu.z - xv.z;
        // quadratic bending, relative form
        fx -= w * dx;
        fy -= w * dy;
        fz -= w * dz;
        if (L >= 0.f) {
            // mass-spring stretch towards neighbour u (d = x_u - x_v)
            const float l = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), kEps);
            const float inv = 1.f / l;
            const float C = l - L;
            const float kc = ks * C * inv;
            fx += kc * dx;
            fy += kc * dy;
            fz += kc * dz;
            const float xsq = inv * inv;
            const float b = ks * fmaxf(1.f - L * inv, 0.f);
            const float c = ks * xsq - b * xsq;
            h00 += c * dx * dx + b;
            h01 += c * dx * dy;
            h02 += c * dx * dz;
            h11 += c * dy * dy + b;
            h12 += c * dy * dz;
            h22 += c * dz * dz + b;
        }
    }
    // reduce the TPV lanes of a vertex
#pragma unroll
    for (int o = TPV / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        h00 += __shfl_xor_sync(0xffffffffu, h00, o);
        h01 += __shfl_xor_sync(0xffffffffu, h01, o);
        h02 += __shfl_xor_sync(0xffffffffu, h02, o);
        h11 += __shfl_xor_sync(0xffffffffu, h11, o);
        h12 += __shfl_xor_sync(0xffffffffu, h12, o);
        h22 += __shfl_xor_sync(0xffffffffu, h22, o);
    }
    if (!active || (lane % TPV) != 0) return;

    // inertia: H += m/h^2 I (+1e9 I pinned), f += -m/h^2 ((x - x0) - v h) + m a
    const float4 p0 = __ldg(&a.x0[v]);
    const float4 vv = __ldg(&a.vel[v]);
    const float4 acc = __ldg(&a.accel[__float_as_int(vv.w)]);
    const float m = p0.w;
    const float mh = m * a.h2inv;
    fx += -mh * ((xv.x - p0.x) - vv.x * a.h) + m * acc.x;
    fy += -mh * ((xv.y - p0.y) - vv.y * a.h) + m * acc.y;
    fz += -mh * ((xv.z - p0.z) - vv.z * a.h) + m * acc.z;
    const float dg = mh + mv.y + mv.x;
    h00 += dg;
    h11 += dg;
    h22 += dg;

    // symmetric 3x3 solve by adjugate / determinant
    const float c00 = h11 * h22 - h12 * h12;
    const float c01 = h02 * h12 - h01 * h22;
    const float c02 = h01 * h12 - h02 * h11;
    const float det = h00 * c00 + h01 * c01 + h02 * c02;
    if (fabsf(det) > kEps) {
        const float c11 = h00 * h22 - h02 * h02;
        const float c12 = h01 * h02 - h00 * h12;
        const float c22 = h00 * h11 - h01 * h01;
        const float id = 1.f / det;
        float4 xn = xv;
        xn.x += (c00 * fx + c01 * fy + c02 * fz) * id;
        xn.y += (c01 * fx + c11 * fy + c12 * fz) * id;
        xn.z += (c02 * fx + c12 * fy + c22 * fz) * id;
        a.x[v] = xn;
    }
}

}  // namespace ats
