// ats_kernels.cuh -- the VBD colour-sweep kernel (sm_100a).
//
// Data layout in HBM (float4 = 16 B, one 128-bit load per vertex record):
//   x     [V]  current iterate, w unused
//   x0    [V]  frame / substep start position, w = mass
//   vel   [V]  velocity, w = the vertex's bending Hessian diagonal (a copy of vm.x)
//   vm    [V]  {k_b * sum Q_oo (bending Hessian diagonal), pin boost (0 / 1e9), inverse mass, instance id bits}
//   inst  [I]  per instance {external acceleration xyz, k_stretch}
// Vertices are ordered instance-major then colour-major, so the vertices of one
// colour of one instance are contiguous and every own-vertex access of a sweep is
// coalesced. The neighbour stencil of a vertex (1-ring plus the far corners of its
// bending edges) is stored sliced-ELL: a slice is one warp, 32/TPV vertices with
// TPV lanes each; row r of a slice is 32 consecutive entries, entry (r, lane) is
// slot r*TPV + lane%TPV of vertex lane/TPV. The first "edge rows" hold the
// neighbours joined by an edge ({index, bending weight} 8 B + rest length 4 B), the
// remaining rows the bending-only neighbours ({index, weight} 8 B), so a row is one
// or two coalesced loads and the spring math is skipped warp-uniformly on
// bending-only rows.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ats {

constexpr float kEps = 1.19209290E-7f;  // src/SharedDefine/constant_value.h:9
constexpr float kPinBoost = 1e9f;       // Hessian boost of a pinned vertex (vm.y), xpbd_constraints.h:4058

// Position access of the sweep and XPBD bodies: plain loads / stores in kernels that
// end at each colour (a launch starts with a clean L1), L2-only ones in the persistent
// kernels, whose blocks read vertices that other SMs wrote since the last grid barrier.
struct PlainMem {
    static __device__ __forceinline__ float4 ld(const float4* p) { return *p; }
    static __device__ __forceinline__ void st(float4* p, float4 v) { *p = v; }
};
struct L2Mem {
    static __device__ __forceinline__ float4 ld(const float4* p) { return __ldcg(p); }
    static __device__ __forceinline__ void st(float4* p, float4 v) { __stcg(p, v); }
};
struct SweepArgs {
    float4* __restrict__ x;
    const float4* __restrict__ x0;
    const float4* __restrict__ vel;
    const float4* __restrict__ vm;
    const int2* __restrict__ st_iw;
    const float* __restrict__ st_rest;
    const int4* __restrict__ slices;
    const int* __restrict__ slice_inst;  // instance of each slice
    const int2* __restrict__ slice_meta; // {instance, pinned-vertex bits} of each slice
    const float4* __restrict__ inst;
    const int* __restrict__ active;      // vbd_sweep_kernel: per instance, null = all active
    const int* __restrict__ list;        // vbd_sweep_list_kernel: this colour's active slices
    const int* __restrict__ list_count;  // and their number (device)
    int slice_begin, slice_end;
    float h, h2inv;
};

// Programmatic dependent launch: a sweep may start while the previous sweep of the
// stream drains; everything it reads before grid_dependency_wait() is constant for
// the life of the handle (stencil, slices, per-vertex material, instance table),
// everything after it (x, x0, vel) is ordered behind the previous kernel.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependent_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Adds the spring to neighbour u (d = x_u - x_v, rest length L) and the bending
// term -w d to the force f and the symmetric Hessian h:
// f += k C d / l, He = k/l^2 d d^T + k max(1 - L/l, 0) (I - d d^T / l^2),
// with l = max(|d|, FLT_EPSILON) as VBD::compute_stretch_mass_spring.
// Every operation is an explicitly rounded intrinsic (fmaf / __fmul_rn / __fadd_rn),
// which the compiler never fuses or reorders: the sweep kernels, whatever their
// launch shape, compute bit-identical results.
__device__ __forceinline__ void vbd_edge(float4 xv, float4 xu, float L, float w, float ks, float& fx, float& fy,
                                         float& fz, float& h00, float& h01, float& h02, float& h11, float& h12,
                                         float& h22) {
    const float dx = __fsub_rn(xu.x, xv.x), dy = __fsub_rn(xu.y, xv.y), dz = __fsub_rn(xu.z, xv.z);
    fx = fmaf(-w, dx, fx);
    fy = fmaf(-w, dy, fy);
    fz = fmaf(-w, dz, fz);
    if (L >= 0.f) {
        const float l2 = fmaf(dx, dx, fmaf(dy, dy, __fmul_rn(dz, dz)));
        const float inv = rsqrtf(fmaxf(l2, kEps * kEps));
        const float l = fmaxf(__fmul_rn(l2, inv), kEps);
        const float kc = __fmul_rn(__fmul_rn(ks, __fsub_rn(l, L)), inv);
        fx = fmaf(kc, dx, fx);
        fy = fmaf(kc, dy, fy);
        fz = fmaf(kc, dz, fz);
        const float xsq = __fmul_rn(inv, inv);
        const float b = __fmul_rn(ks, fmaxf(fmaf(-L, inv, 1.f), 0.f));
        const float c = __fmul_rn(__fsub_rn(ks, b), xsq);
        const float cx = __fmul_rn(c, dx), cy = __fmul_rn(c, dy);
        h00 = __fadd_rn(h00, fmaf(cx, dx, b));
        h01 = fmaf(cx, dy, h01);
        h02 = fmaf(cx, dz, h02);
        h11 = __fadd_rn(h11, fmaf(cy, dy, b));
        h12 = fmaf(cy, dz, h12);
        h22 = __fadd_rn(h22, fmaf(__fmul_rn(c, dz), dz, b));
    }
}

// Bending-only neighbour: quadratic bending in relative coordinates, -w (x_u - x_v).
__device__ __forceinline__ void vbd_bend(float4 xv, float4 xu, float w, float& fx, float& fy, float& fz) {
    fx = fmaf(-w, __fsub_rn(xu.x, xv.x), fx);
    fy = fmaf(-w, __fsub_rn(xu.y, xv.y), fy);
    fz = fmaf(-w, __fsub_rn(xu.z, xv.z), fz);
}

// The per-vertex part of a sweep, shared by both sweep kernels: the RE + RB gathered
// neighbours (rows beyond them go through loops), the lane reduction, inertia and the
// guarded 3x3 solve; the leader lane of a vertex writes x.
template <int TPV, int RE, int RB, class M = PlainMem>
__device__ __forceinline__ void sweep_vertex(const SweepArgs& a, int v, bool leader, int base, int bbase, int erows,
                                             int brows, float4 xv, const float4 (&xe)[RE], const float (&le)[RE],
                                             const float (&we)[RE], const float4 (&xb)[RB], const float (&wb)[RB],
                                             float ks, float4 ip, float4 mv, float4 p0, float4 vv) {
    float fx = 0.f, fy = 0.f, fz = 0.f;
    float h00 = 0.f, h01 = 0.f, h02 = 0.f, h11 = 0.f, h12 = 0.f, h22 = 0.f;
#pragma unroll
    for (int r = 0; r < RE; ++r) vbd_edge(xv, xe[r], le[r], we[r], ks, fx, fy, fz, h00, h01, h02, h11, h12, h22);
    for (int r = RE; r < erows; ++r) {
        const int2 iw = __ldg(&a.st_iw[base + r * 32]);
        vbd_edge(xv, M::ld(&a.x[iw.x]), __ldg(&a.st_rest[base + r * 32]), __int_as_float(iw.y), ks, fx, fy, fz, h00, h01, h02,
                 h11, h12, h22);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) vbd_bend(xv, xb[r], wb[r], fx, fy, fz);
    for (int r = RB; r < brows; ++r) {
        const int2 iw = __ldg(&a.st_iw[bbase + r * 32]);
        vbd_bend(xv, M::ld(&a.x[iw.x]), __int_as_float(iw.y), fx, fy, fz);
    }
    // reduce the TPV lanes of a vertex
#pragma unroll
    for (int o = TPV / 2; o > 0; o >>= 1) {
        fx = __fadd_rn(fx, __shfl_xor_sync(0xffffffffu, fx, o));
        fy = __fadd_rn(fy, __shfl_xor_sync(0xffffffffu, fy, o));
        fz = __fadd_rn(fz, __shfl_xor_sync(0xffffffffu, fz, o));
        h00 = __fadd_rn(h00, __shfl_xor_sync(0xffffffffu, h00, o));
        h01 = __fadd_rn(h01, __shfl_xor_sync(0xffffffffu, h01, o));
        h02 = __fadd_rn(h02, __shfl_xor_sync(0xffffffffu, h02, o));
        h11 = __fadd_rn(h11, __shfl_xor_sync(0xffffffffu, h11, o));
        h12 = __fadd_rn(h12, __shfl_xor_sync(0xffffffffu, h12, o));
        h22 = __fadd_rn(h22, __shfl_xor_sync(0xffffffffu, h22, o));
    }
    if (!leader) return;

    // inertia: H += m/h^2 I (+1e9 I pinned), f += -m/h^2 ((x - x0) - v h) + m a
    const float m = p0.w;
    const float mh = __fmul_rn(m, a.h2inv);
    fx = __fadd_rn(fx, fmaf(-mh, fmaf(-vv.x, a.h, __fsub_rn(xv.x, p0.x)), __fmul_rn(m, ip.x)));
    fy = __fadd_rn(fy, fmaf(-mh, fmaf(-vv.y, a.h, __fsub_rn(xv.y, p0.y)), __fmul_rn(m, ip.y)));
    fz = __fadd_rn(fz, fmaf(-mh, fmaf(-vv.z, a.h, __fsub_rn(xv.z, p0.z)), __fmul_rn(m, ip.z)));
    const float dg = __fadd_rn(__fadd_rn(mh, mv.y), mv.x);
    h00 = __fadd_rn(h00, dg);
    h11 = __fadd_rn(h11, dg);
    h22 = __fadd_rn(h22, dg);

    // symmetric 3x3 solve by adjugate / determinant, guarded by |det| > FLT_EPSILON
    const float c00 = fmaf(h11, h22, -__fmul_rn(h12, h12));
    const float c01 = fmaf(h02, h12, -__fmul_rn(h01, h22));
    const float c02 = fmaf(h01, h12, -__fmul_rn(h02, h11));
    const float det = fmaf(h00, c00, fmaf(h01, c01, __fmul_rn(h02, c02)));
    if (fabsf(det) > kEps) {
        const float c11 = fmaf(h00, h22, -__fmul_rn(h02, h02));
        const float c12 = fmaf(h01, h02, -__fmul_rn(h00, h12));
        const float c22 = fmaf(h00, h11, -__fmul_rn(h01, h01));
        const float id = __fdiv_rn(1.f, det);
        float4 xn = xv;
        xn.x = fmaf(fmaf(c00, fx, fmaf(c01, fy, __fmul_rn(c02, fz))), id, xv.x);
        xn.y = fmaf(fmaf(c01, fx, fmaf(c11, fy, __fmul_rn(c12, fz))), id, xv.y);
        xn.z = fmaf(fmaf(c02, fx, fmaf(c12, fy, __fmul_rn(c22, fz))), id, xv.z);
        M::st(&a.x[v], xn);
    }
}

// One VBD colour sweep: for every vertex of the colour, inertia + mass-spring
// stretch + quadratic bending gradient and Hessian (reference:
// VBD::compute_inertia / compute_stretch_mass_spring / compute_bending_quadratic,
// xpbd_constraints.h:4027-4205), then the determinant-guarded 3x3 solve of
// example2_async_iter.cpp:993-1014, all in registers (Hf never goes to memory).
// Bending is linear in x, so the per-bending-edge terms -k_b sum_j Q[o][j] x_j are
// merged per (vertex, neighbour) into one weight W and applied in relative
// coordinates, the same force because every row of Q sums to zero.
// RE edge rows and RB bending rows are loaded up front (all stencil entries, then
// all gathers) so that a thread has RE + RB independent loads in flight; rows
// beyond them go through loops.
template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(256) vbd_sweep_kernel(SweepArgs a) {
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int slice = a.slice_begin + warp;
    const int lane = threadIdx.x & 31;
    if (slice >= a.slice_end) {
        grid_dependency_wait();
        allow_dependent_launch();
        return;
    }
    const int4 sd = __ldg(&a.slices[slice]);  // vbegin, nverts, entry offset, rows | edge rows << 16
    const int rows = sd.w & 0xffff, erows = sd.w >> 16, brows = rows - erows;
    const int k = lane / TPV;
    const bool leader = k < sd.y && (lane % TPV) == 0;
    const int v = sd.x + min(k, sd.y - 1);
    const int base = sd.z + lane;
    const int bbase = base + erows * 32;

    // With an activity mask (written by the kernel before) the flag is read first,
    // after the dependency wait, so that a converged instance costs one load per
    // slice; without one, the constant data below is fetched before the wait.
    if (a.active) {
        grid_dependency_wait();
        allow_dependent_launch();
        if (!a.active[__ldg(&a.slice_inst[slice])]) return;
    }
    // constant data: stencil rows, material, instance parameters
    int ue[RE], ub[RB];
    float we[RE], le[RE], wb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) {
        ue[r] = v;
        we[r] = 0.f;
        le[r] = -1.f;
        if (r < erows) {
            const int2 iw = __ldg(&a.st_iw[base + r * 32]);
            ue[r] = iw.x;
            we[r] = __int_as_float(iw.y);
            le[r] = __ldg(&a.st_rest[base + r * 32]);
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        ub[r] = v;
        wb[r] = 0.f;
        if (r < brows) {
            const int2 iw = __ldg(&a.st_iw[bbase + r * 32]);
            ub[r] = iw.x;
            wb[r] = __int_as_float(iw.y);
        }
    }
    const float4 mv = __ldg(&a.vm[v]);
    const float4 ip = __ldg(&a.inst[__float_as_int(mv.w)]);
    const float ks = ip.w;

    if (!a.active) {
        grid_dependency_wait();
        allow_dependent_launch();
    }

    // positions and frame-start state (ordered behind the previous kernel); the
    // neighbours belong to other colours, which this launch does not write
    const float4 xv = a.x[v];
    float4 xe[RE], xb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) xe[r] = a.x[ue[r]];
#pragma unroll
    for (int r = 0; r < RB; ++r) xb[r] = a.x[ub[r]];
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), vv = p0;
    if (leader) {
        p0 = a.x0[v];
        vv = a.vel[v];
    }

    sweep_vertex<TPV, RE, RB>(a, v, leader, base, bbase, erows, brows, xv, xe, le, we, xb, wb, ks, ip, mv, p0, vv);
}

// Loads of the data a sweep reads once per iteration and never writes (stencil rows,
// rest lengths, vertex records, frame-start state): through the read-only path, or
// as streaming loads (ld.global.cs: evict-first in L1 and L2), which leave L2 to
// the positions that every colour's sweep gathers again.
struct ConstLoads {
    template <class T>
    static __device__ __forceinline__ T ld(const T* p) { return __ldg(p); }
};
struct StreamLoads {
    template <class T>
    static __device__ __forceinline__ T ld(const T* p) { return __ldcs(p); }
};

// One slice of a sweep (descriptor sd): every vertex of the slice (its constant data,
// then all neighbour positions at once, then the solve). M chooses how positions are
// accessed, LD how the per-iteration constant data is loaded. With META the material
// record vm is not read: the instance and the pinned vertices come from the slice's
// metadata meta = {instance, pinned bits}, the bending diagonal from vel.w (the same
// values, 16 bytes less per vertex).
template <int TPV, int RE, int RB, class M, class LD = ConstLoads, bool META = false>
__device__ __forceinline__ void sweep_slice_sd(const SweepArgs& a, int4 sd, int lane, int2 meta = make_int2(0, 0)) {
    const int rows = sd.w & 0xffff, erows = sd.w >> 16, brows = rows - erows;
    const int k = lane / TPV;
    const bool leader = k < sd.y && (lane % TPV) == 0;
    const int v = sd.x + min(k, sd.y - 1);
    const int base = sd.z + lane;
    const int bbase = base + erows * 32;
    int ue[RE], ub[RB];
    float we[RE], le[RE], wb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) {
        ue[r] = v;
        we[r] = 0.f;
        le[r] = -1.f;
        if (r < erows) {
            const int2 iw = LD::ld(&a.st_iw[base + r * 32]);
            ue[r] = iw.x;
            we[r] = __int_as_float(iw.y);
            le[r] = LD::ld(&a.st_rest[base + r * 32]);
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        ub[r] = v;
        wb[r] = 0.f;
        if (r < brows) {
            const int2 iw = LD::ld(&a.st_iw[bbase + r * 32]);
            ub[r] = iw.x;
            wb[r] = __int_as_float(iw.y);
        }
    }
    float4 mv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!META) mv = LD::ld(&a.vm[v]);
    const float4 ip = __ldg(&a.inst[META ? meta.x : __float_as_int(mv.w)]);
    const float4 xv = M::ld(&a.x[v]);
    float4 xe[RE], xb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) xe[r] = M::ld(&a.x[ue[r]]);
#pragma unroll
    for (int r = 0; r < RB; ++r) xb[r] = M::ld(&a.x[ub[r]]);
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), vv = p0;
    if (leader) {
        p0 = LD::ld(&a.x0[v]);
        vv = LD::ld(&a.vel[v]);
    }
    if (META) mv = make_float4(vv.w, ((unsigned)meta.y >> k) & 1u ? kPinBoost : 0.f, 0.f, 0.f);
    sweep_vertex<TPV, RE, RB, M>(a, v, leader, base, bbase, erows, brows, xv, xe, le, we, xb, wb, ip.w, ip, mv, p0,
                                 vv);
}

template <int TPV, int RE, int RB, class M>
__device__ __forceinline__ void sweep_slice(const SweepArgs& a, int slice, int lane) {
    sweep_slice_sd<TPV, RE, RB, M>(a, __ldg(&a.slices[slice]), lane);
}

// ---------------------------------------------------------------- pipelined list sweep
// A warp's slices are independent of one another inside a colour: a slice reads its own
// vertices' records, its stencil and the positions of neighbours of other colours, none
// of which this colour writes. So while a warp computes one slice, the constant data of
// its next slice (stencil rows, rest lengths, the lanes' own vertex records) is already
// on its way into shared memory by cp.async, and the descriptor of the slice after that
// is loading into registers. Every lane stages and later reads only its own entries.
template <int RE, int RB>
struct SliceStage {
    int2 iw[RE + RB][32];  // stencil rows: {neighbour, bending weight}
    float rest[RE][32];    // rest lengths of the edge rows
    float4 vm[32], x0[32], vel[32];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int TPV, int RE, int RB>
__device__ __forceinline__ void stage_slice(SliceStage<RE, RB>& S, const SweepArgs& a, int4 sd, int lane) {
    const int rows = sd.w & 0xffff, erows = sd.w >> 16, brows = rows - erows;
    const int v = sd.x + min(lane / TPV, sd.y - 1);
    const int base = sd.z + lane, bbase = base + erows * 32;
#pragma unroll
    for (int r = 0; r < RE; ++r)
        if (r < erows) {
            cp_async8(&S.iw[r][lane], &a.st_iw[base + r * 32]);
            cp_async4(&S.rest[r][lane], &a.st_rest[base + r * 32]);
        }
#pragma unroll
    for (int r = 0; r < RB; ++r)
        if (r < brows) cp_async8(&S.iw[RE + r][lane], &a.st_iw[bbase + r * 32]);
    cp_async16(&S.vm[lane], &a.vm[v]);
    cp_async16(&S.x0[lane], &a.x0[v]);
    cp_async16(&S.vel[lane], &a.vel[v]);
}

// sweep_slice with the constant data from a staged slice
template <int TPV, int RE, int RB>
__device__ __forceinline__ void sweep_staged(const SweepArgs& a, const SliceStage<RE, RB>& S, int4 sd, int lane) {
    const int rows = sd.w & 0xffff, erows = sd.w >> 16, brows = rows - erows;
    const int k = lane / TPV;
    const bool leader = k < sd.y && (lane % TPV) == 0;
    const int v = sd.x + min(k, sd.y - 1);
    const int base = sd.z + lane;
    const int bbase = base + erows * 32;
    int ue[RE], ub[RB];
    float we[RE], le[RE], wb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) {
        ue[r] = v;
        we[r] = 0.f;
        le[r] = -1.f;
        if (r < erows) {
            const int2 iw = S.iw[r][lane];
            ue[r] = iw.x;
            we[r] = __int_as_float(iw.y);
            le[r] = S.rest[r][lane];
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        ub[r] = v;
        wb[r] = 0.f;
        if (r < brows) {
            const int2 iw = S.iw[RE + r][lane];
            ub[r] = iw.x;
            wb[r] = __int_as_float(iw.y);
        }
    }
    const float4 mv = S.vm[lane];
    const float4 ip = __ldg(&a.inst[__float_as_int(mv.w)]);
    const float4 xv = a.x[v];
    float4 xe[RE], xb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) xe[r] = a.x[ue[r]];
#pragma unroll
    for (int r = 0; r < RB; ++r) xb[r] = a.x[ub[r]];
    sweep_vertex<TPV, RE, RB, PlainMem>(a, v, leader, base, bbase, erows, brows, xv, xe, le, we, xb, wb, ip.w, ip, mv,
                                        S.x0[lane], S.vel[lane]);
}

// The list sweep, software-pipelined across each warp's slices (two shared-memory
// stages per warp, dynamic shared memory 2 * warps per block * sizeof(SliceStage)).
template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(256) vbd_sweep_pipe_kernel(SweepArgs a) {
    extern __shared__ __align__(16) unsigned char pipe_smem[];
    grid_dependency_wait();  // the list and the positions come from the kernels before
    allow_dependent_launch();
    const int lane = threadIdx.x & 31;
    SliceStage<RE, RB>* buf = reinterpret_cast<SliceStage<RE, RB>*>(pipe_smem) + 2 * (threadIdx.x >> 5);
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int count = *a.list_count;
    int idx = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (idx >= count) return;
    int4 sd_cur = __ldg(&a.slices[a.list[idx]]);
    stage_slice<TPV, RE, RB>(buf[0], a, sd_cur, lane);
    cp_async_commit();
    int4 sd_nxt = make_int4(0, 0, 0, 0);
    if (idx + nwarps < count) sd_nxt = __ldg(&a.slices[a.list[idx + nwarps]]);
    for (int it = 0; idx < count; idx += nwarps, ++it) {
        const int cur = it & 1;
        if (idx + nwarps < count) stage_slice<TPV, RE, RB>(buf[cur ^ 1], a, sd_nxt, lane);
        cp_async_commit();  // empty when there is no next slice: the wait below stays uniform
        int4 sd_after = make_int4(0, 0, 0, 0);
        if (idx + 2 * nwarps < count) sd_after = __ldg(&a.slices[a.list[idx + 2 * nwarps]]);
        cp_async_wait<1>();  // the current slice's stage has landed
        sweep_staged<TPV, RE, RB>(a, buf[cur], sd_cur, lane);
        __syncwarp();  // this stage is refilled two slices later
        sd_cur = sd_nxt;
        sd_nxt = sd_after;
    }
    cp_async_wait<0>();
}

// The sweep of a residual-driven frame: only the slices of instances still iterating,
// listed per colour by the compaction after each probe (order within a colour does not
// matter: its vertices are independent). A grid of resident size strides over the
// list, so a converged instance costs nothing, not even a CTA launch.
template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(256) vbd_sweep_list_kernel(SweepArgs a) {
    grid_dependency_wait();  // the list and the positions come from the kernels before
    allow_dependent_launch();
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int count = *a.list_count;
    for (int idx = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); idx < count; idx += nwarps)
        sweep_slice<TPV, RE, RB, PlainMem>(a, a.list[idx], lane);
}

// The list sweep with streaming loads for the per-iteration constant data and the
// next slice's descriptor and metadata in flight while the current slice computes: a
// warp loads the list entry two slices ahead and the descriptor one slice ahead, so
// the chain in front of each slice's neighbour gathers is its stencil rows alone. The
// material record is not read (sweep_slice_sd with META).
template <int TPV, int RE, int RB>
__device__ __forceinline__ void stream_sweep(const SweepArgs& a) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int count = *a.list_count;
    int idx = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (idx >= count) return;
    const int first = a.list[idx];
    int4 sd = __ldg(&a.slices[first]);
    int2 meta = __ldg(&a.slice_meta[first]);
    int next = idx + nwarps < count ? a.list[idx + nwarps] : 0;
    for (;;) {
        const bool more = idx + nwarps < count;
        int4 sd_next = sd;
        int2 meta_next = meta;
        if (more) {
            sd_next = __ldg(&a.slices[next]);
            meta_next = __ldg(&a.slice_meta[next]);
        }
        const int after = idx + 2 * nwarps < count ? a.list[idx + 2 * nwarps] : 0;
        sweep_slice_sd<TPV, RE, RB, PlainMem, StreamLoads, true>(a, sd, lane, meta);
        if (!more) break;
        idx += nwarps;
        sd = sd_next;
        meta = meta_next;
        next = after;
    }
}

template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(256) vbd_sweep_stream_kernel(SweepArgs a) {
    grid_dependency_wait();  // the list and the positions come from the kernels before
    allow_dependent_launch();
    stream_sweep<TPV, RE, RB>(a);
}

}  // namespace ats
