// ats_cloth.cu -- solver handle, sm_100a kernels and the C ABI of libats_b200.so.
//
// Each step entry point is one launcher task of the reference
// (src/heterogeneous/launcher.h FunctionID); a frame is the loop of
// CpuSolver::physics_step_vbd / physics_step_xpbd (examples/example2_async_iter.cpp:
// 1017-1143) issued as kernels on one stream, optionally replayed as a CUDA graph.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include "ats_internal.cuh"
#include "ats_kernels.cuh"
#include "ats_umma.cuh"

namespace ats {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_kernel_launches{0};
static std::mutex g_graph_mu;
static std::unordered_map<cudaGraphExec_t, int> g_graph_kernels;

void count_launch(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void register_graph(cudaGraphExec_t exec, cudaGraph_t g) {
    size_t n = 0;
    int kernels = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess && n > 0) {
        std::vector<cudaGraphNode_t> nodes(n);
        if (cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
            for (size_t i = 0; i < n; ++i) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
            }
    }
    std::lock_guard<std::mutex> lock(g_graph_mu);
    g_graph_kernels[exec] = kernels;
}

void count_graph_launch(cudaGraphExec_t exec) {
    int k = 0;
    {
        std::lock_guard<std::mutex> lock(g_graph_mu);
        auto it = g_graph_kernels.find(exec);
        if (it != g_graph_kernels.end()) k = it->second;
    }
    g_kernel_launches.fetch_add(k, std::memory_order_relaxed);
}

namespace {

// ---------------------------------------------------------------- kernels

// Explicitly rounded FP32 operations: the predict / update / XPBD kernels evaluate
// every term in the order of the reference's CPU code with no fused multiply-add,
// so they round exactly as the CPU restatement does.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdot(float3 a, float3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }

// Core::predict_position (xpbd_constraints.h:321-384): v_pred = v + h a (0 if pinned),
// x = x0 + h v_pred.
__global__ void predict_kernel(float4* __restrict__ x, const float4* __restrict__ x0, const float4* __restrict__ vel,
                               const float4* __restrict__ vm, const float4* __restrict__ inst, int n, float h) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = x0[i], v = vel[i], m = vm[i];
    float4 a = __ldg(&inst[__float_as_int(m.w)]);
    bool pinned = m.y != 0.f;
    float vx = fa(v.x, fm(h, a.x)), vy = fa(v.y, fm(h, a.y)), vz = fa(v.z, fm(h, a.z));
    if (pinned) vx = vy = vz = 0.f;
    x[i] = make_float4(fa(p.x, fm(h, vx)), fa(p.y, fm(h, vy)), fa(p.z, fm(h, vz)), 0.f);
}

// Core::update_velocity (xpbd_constraints.h:535-581): v = (x - x0)/h * damp, x0 = x.
__global__ void update_kernel(const float4* __restrict__ x, float4* __restrict__ x0, float4* __restrict__ vel, int n,
                              float h, float damp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = x[i], q = x0[i], v = vel[i];
    v.x = fm(fs(p.x, q.x) / h, damp);
    v.y = fm(fs(p.y, q.y) / h, damp);
    v.z = fm(fs(p.z, q.z) / h, damp);
    vel[i] = v;
    x0[i] = make_float4(p.x, p.y, p.z, q.w);
}

// The constant data of one stretch constraint: vertex ids, rest length, stiffness and
// the endpoints' inverse masses.
struct StretchConst {
    int2 ed;
    float L, k, w0, w1;
};
__device__ __forceinline__ StretchConst load_stretch(int i, const float4* __restrict__ vm, const int2* __restrict__ edge,
                                                     const float* __restrict__ rest, const float* __restrict__ kst) {
    StretchConst c;
    c.ed = __ldg(&edge[i]);
    c.L = __ldg(&rest[i]);
    c.k = __ldg(&kst[i]);
    c.w0 = __ldg(&vm[c.ed.x]).z;
    c.w1 = __ldg(&vm[c.ed.y]).z;
    return c;
}

// solve_stretch_mass_spring_template (xpbd_constraints.h:984-1059) for constraint i.
template <class M>
__device__ __forceinline__ void solve_stretch(float4* __restrict__ x, float* __restrict__ lambda, int i,
                                              const StretchConst& c, float h) {
    const float4 p0 = M::ld(&x[c.ed.x]), p1 = M::ld(&x[c.ed.y]);
    const float lam = lambda[i];
    const float3 d = make_float3(fs(p1.x, p0.x), fs(p1.y, p0.y), fs(p1.z, p0.z));
    const float lsq = fdot(d, d);
    if ((double)lsq < 1e-8) return;
    const float l = sqrtf(lsq);
    const float C = fs(l, c.L);
    const float gx = -(d.x / l), gy = -(d.y / l), gz = -(d.z / l);
    const float alpha = c.k < kEps ? 1e9f : 1.f / fm(fm(c.k, h), h);
    const float denom = fa(alpha, fa(c.w0, c.w1));
    const float dl = fs(-C, fm(alpha, lam)) / denom;
    lambda[i] = fa(lam, dl);
    if (denom != 0.f) {
        const float s0 = fm(dl, c.w0), s1 = fm(-dl, c.w1);
        M::st(&x[c.ed.x], make_float4(fa(p0.x, fm(s0, gx)), fa(p0.y, fm(s0, gy)), fa(p0.z, fm(s0, gz)), p0.w));
        M::st(&x[c.ed.y], make_float4(fa(p1.x, fm(s1, gx)), fa(p1.y, fm(s1, gy)), fa(p1.z, fm(s1, gz)), p1.w));
    }
}

// The constant data of one bending constraint: vertex ids, the 10 unique entries of
// the symmetric Q and k_b, and the inverse masses.
struct BendConst {
    int4 id;
    float4 qa, qb, qc;
    float w[4];
};
__device__ __forceinline__ BendConst load_bend(int i, const float4* __restrict__ vm, const int4* __restrict__ idx,
                                               const float4* __restrict__ q) {
    BendConst c;
    c.id = __ldg(&idx[i]);
    c.qa = __ldg(&q[3 * i]);
    c.qb = __ldg(&q[3 * i + 1]);
    c.qc = __ldg(&q[3 * i + 2]);
    c.w[0] = __ldg(&vm[c.id.x]).z;
    c.w[1] = __ldg(&vm[c.id.y]).z;
    c.w[2] = __ldg(&vm[c.id.z]).z;
    c.w[3] = __ldg(&vm[c.id.w]).z;
    return c;
}

// solve_bending_quadratic_template (xpbd_constraints.h:1170-1229, core :1062-1126,
// get_delta_xpbd_4 :211-236) for constraint i.
template <class M>
__device__ __forceinline__ void solve_bend(float4* __restrict__ x, float* __restrict__ lambda, int i,
                                           const BendConst& c, float h) {
    float Q[4][4];
    Q[0][0] = c.qa.x; Q[0][1] = Q[1][0] = c.qa.y; Q[0][2] = Q[2][0] = c.qa.z; Q[0][3] = Q[3][0] = c.qa.w;
    Q[1][1] = c.qb.x; Q[1][2] = Q[2][1] = c.qb.y; Q[1][3] = Q[3][1] = c.qb.z; Q[2][2] = c.qb.w;
    Q[2][3] = Q[3][2] = c.qc.x; Q[3][3] = c.qc.y;
    const float kb = c.qc.z;
    const int vid[4] = {c.id.x, c.id.y, c.id.z, c.id.w};
    float3 p[4];
    float pw[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float4 t = M::ld(&x[vid[j]]);
        p[j] = make_float3(t.x, t.y, t.z);
        pw[j] = t.w;
    }
    // C = 1/2 sum_ij Q_ij <x_i, x_j>
    float sum = 0.f;
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) sum = fa(sum, fm(Q[ii][jj], fdot(p[ii], p[jj])));
    const float C = fm(0.5f, sum);
    // gradient_i = sum_j Q_ij x_j (the negated force of the reference)
    float3 g[4];
    float denom = 0.f;
#pragma unroll
    for (int ii = 0; ii < 4; ++ii) {
        float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            gx = fa(gx, fm(Q[ii][jj], p[jj].x));
            gy = fa(gy, fm(Q[ii][jj], p[jj].y));
            gz = fa(gz, fm(Q[ii][jj], p[jj].z));
        }
        g[ii] = make_float3(gx, gy, gz);
        denom = fa(denom, fm(c.w[ii], fdot(g[ii], g[ii])));
    }
    const float alpha = kb < kEps ? 1e12f : 1.f / fm(fm(kb, h), h);
    denom = fa(denom, alpha);
    const float lam = lambda[i];
    const float dl = fs(-C, fm(alpha, lam)) / denom;
    lambda[i] = fa(lam, dl);
    if (denom != 0.f) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float s = fm(dl, c.w[j]);
            M::st(&x[vid[j]],
                  make_float4(fa(p[j].x, fm(s, g[j].x)), fa(p[j].y, fm(s, g[j].y)), fa(p[j].z, fm(s, g[j].z)), pw[j]));
        }
    }
}

// One stretch colour. Programmatic dependent launch: the constraint's constant data is
// loaded before the wait on the previous colour; positions and lambda after it.
__global__ void xpbd_stretch_kernel(float4* __restrict__ x, const float4* __restrict__ vm, const int2* __restrict__ edge,
                                    const float* __restrict__ rest, const float* __restrict__ kst,
                                    float* __restrict__ lambda, int b, int e, float h) {
    const int i = b + blockIdx.x * blockDim.x + threadIdx.x;
    StretchConst c = {};
    if (i < e) c = load_stretch(i, vm, edge, rest, kst);
    grid_dependency_wait();
    allow_dependent_launch();
    if (i < e) solve_stretch<PlainMem>(x, lambda, i, c, h);
}

// One bending colour (as xpbd_stretch_kernel).
__global__ void xpbd_bending_kernel(float4* __restrict__ x, const float4* __restrict__ vm, const int4* __restrict__ idx,
                                    const float4* __restrict__ q, float* __restrict__ lambda, int b, int e, float h) {
    const int i = b + blockIdx.x * blockDim.x + threadIdx.x;
    BendConst c = {};
    if (i < e) c = load_bend(i, vm, idx, q);
    grid_dependency_wait();
    allow_dependent_launch();
    if (i < e) solve_bend<PlainMem>(x, lambda, i, c, h);
}

// Grid-wide barrier of the persistent kernels, whose blocks are co-resident (a
// cooperative launch). bar[0] counts the arrivals since the launch (set to 0 before
// it); barrier k of the launch is passed once the count reaches k * gridDim.x, which
// each block tracks in `target`, so an arrival is one atomic and nothing is reset.
// Thread 0 of every block publishes the block's writes (device-scope fence), arrives,
// and polls the count with acquire loads (back to back for the first
// kBarrierFastPolls, then with a short sleep). The wait is bounded: after
// kBarrierSpins polls the block sets bit 31 of the count (kBarrierError) and *err,
// and every block leaves the kernel at its next poll. Returns false on error. The
// host keeps every launch below 2^31 arrivals (kMaxLoopArrivals).
constexpr unsigned kBarrierSpins = 1u << 24;
constexpr unsigned kBarrierFastPolls = 1u << 12;
constexpr unsigned kBarrierError = 0x80000000u;
constexpr unsigned long long kMaxLoopArrivals = 0x7fffffffull;
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err, unsigned& target,
                                             unsigned max_polls = kBarrierSpins) {
    __shared__ int s_ok;
    target += gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned v = atomicAdd(bar, 1u) + 1u;
        unsigned spins = 0;
        while ((v & ~kBarrierError) < target && !(v & kBarrierError)) {
            if (++spins > max_polls) {
                v = atomicOr(bar, kBarrierError) | kBarrierError;
                atomicExch(err, 1);
                break;
            }
            if (spins > kBarrierFastPolls) __nanosleep(64);
            v = ld_acquire_gpu(bar);
        }
        __threadfence();
        s_ok = !(v & kBarrierError);
    }
    __syncthreads();
    return s_ok != 0;
}

constexpr int kXpbdLoopThreads = 640;  // one block per SM, up to 96 registers a thread

// `iterations` VBD iterations of every instance in one cooperative launch: each colour
// is a grid-stride loop of warps over the colour's slices (sweep_slice, the body of
// the list sweep, with L2-only position access), colours are separated by
// grid_barrier. The same per-vertex arithmetic as the one-wave and list sweeps, so the
// same positions. The autotuner keeps it only where it measures faster.
template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(256) vbd_loop_kernel(SweepArgs a, const int* __restrict__ color_slices, int ncolors,
                                                       int iterations, unsigned* bar, int* err) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    unsigned target = 0;
    for (int it = 0; it < iterations; ++it)
        for (int c = 0; c < ncolors; ++c) {
            const int b = __ldg(&color_slices[c]), e = __ldg(&color_slices[c + 1]);
            for (int slice = b + w; slice < e; slice += nwarps) sweep_slice<TPV, RE, RB, L2Mem>(a, slice, lane);
            if (!grid_barrier(bar, err, target)) return;
        }
}

struct XpbdLoopArgs {
    float4* x;
    const float4* vm;
    const int2* edge;
    const float* rest;
    const float* kst;
    float* slambda;
    const int4* bidx;
    const float4* bq;
    float* blambda;
    const int* scolor;  // n_scolors + 1 offsets
    const int* bcolor;  // n_bcolors + 1 offsets
    int nsc, nbc, iterations;
    float h;
    unsigned* bar;
    int* err;
};

// `iterations` XPBD iterations (every stretch colour, then every bending colour, as
// the per-colour launches run them) in one cooperative launch: each colour is a
// grid-stride loop, colours are separated by grid_barrier. Each thread loads the
// constant data of its first constraint of the next colour before the barrier, so
// only the position gather waits for the previous colour. Same arithmetic, same
// results as the per-colour kernels.
__global__ void __launch_bounds__(kXpbdLoopThreads, 1) xpbd_loop_kernel(XpbdLoopArgs a) {
    const int stride = gridDim.x * blockDim.x;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int phases = a.nsc + a.nbc;
    if (phases == 0) return;
    auto range = [&](int ph, int& b, int& e) {
        if (ph < a.nsc) {
            b = __ldg(&a.scolor[ph]);
            e = __ldg(&a.scolor[ph + 1]);
        } else {
            b = __ldg(&a.bcolor[ph - a.nsc]);
            e = __ldg(&a.bcolor[ph - a.nsc + 1]);
        }
    };
    StretchConst sc = {};
    BendConst bc = {};
    unsigned target = 0;
    int b, e;
    range(0, b, e);
    if (b + t < e) {
        if (a.nsc > 0) sc = load_stretch(b + t, a.vm, a.edge, a.rest, a.kst);
        else bc = load_bend(b + t, a.vm, a.bidx, a.bq);
    }
    for (int it = 0; it < a.iterations; ++it) {
        for (int ph = 0; ph < phases; ++ph) {
            range(ph, b, e);
            const bool stretch = ph < a.nsc;
            int i = b + t;
            if (i < e) {
                if (stretch) solve_stretch<L2Mem>(a.x, a.slambda, i, sc, a.h);
                else solve_bend<L2Mem>(a.x, a.blambda, i, bc, a.h);
                for (i += stride; i < e; i += stride) {
                    if (stretch) solve_stretch<L2Mem>(a.x, a.slambda, i, load_stretch(i, a.vm, a.edge, a.rest, a.kst), a.h);
                    else solve_bend<L2Mem>(a.x, a.blambda, i, load_bend(i, a.vm, a.bidx, a.bq), a.h);
                }
            }
            // the next colour's first constraint of this thread, ahead of the barrier
            const int nph = ph + 1 < phases ? ph + 1 : 0;
            if (it + 1 < a.iterations || nph != 0) {
                int nb, ne;
                range(nph, nb, ne);
                if (nb + t < ne) {
                    if (nph < a.nsc) sc = load_stretch(nb + t, a.vm, a.edge, a.rest, a.kst);
                    else bc = load_bend(nb + t, a.vm, a.bidx, a.bq);
                }
            }
            if (!grid_barrier(a.bar, a.err, target)) return;
        }
    }
}

// Core::read_and_solve_conflict (xpbd_constraints.h:815-869), this device's iterate
// being "self": with the fork point init, self and other moved by dx_s, dx_o,
//   weight > FLT_EPSILON: both moved -> init + weight (dx_s + dx_o); one moved -> that
//                         one; none -> init;
//   otherwise:            (self + other) / 2;
// the result becomes both the iterate and the new fork point. "Moved" is
// |dx|^2 != 0 in FP32, summed x, y, z in that order; every operation is rounded
// explicitly, in the reference's order.
__global__ void async_merge_kernel(float4* __restrict__ x, float4* __restrict__ begin, const float* __restrict__ other,
                                   const int* __restrict__ to_caller, int n, float weight) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t o = 3 * (size_t)to_caller[i];
    const float4 ps = x[i], init = begin[i];
    const float po[3] = {other[o], other[o + 1], other[o + 2]};
    const float s3[3] = {ps.x, ps.y, ps.z}, b3[3] = {init.x, init.y, init.z};
    float r[3];
    if (weight > kEps) {
        float ds[3], dq[3];
        for (int k = 0; k < 3; ++k) {
            ds[k] = fs(s3[k], b3[k]);
            dq[k] = fs(po[k], b3[k]);
        }
        const bool act_s = fa(fa(fm(ds[0], ds[0]), fm(ds[1], ds[1])), fm(ds[2], ds[2])) != 0.f;
        const bool act_o = fa(fa(fm(dq[0], dq[0]), fm(dq[1], dq[1])), fm(dq[2], dq[2])) != 0.f;
        for (int k = 0; k < 3; ++k) {
            if (act_s && act_o) r[k] = fa(b3[k], fm(weight, fa(ds[k], dq[k])));
            else if (act_s) r[k] = s3[k];
            else if (act_o) r[k] = po[k];
            else r[k] = b3[k];
        }
    } else {
        for (int k = 0; k < 3; ++k) r[k] = fm(0.5f, fa(s3[k], po[k]));
    }
    x[i] = make_float4(r[0], r[1], r[2], ps.w);
    begin[i] = make_float4(r[0], r[1], r[2], 0.f);
}

// State I/O between the caller's vertex order (3 floats per vertex) and the layout.
__global__ void scatter_state_kernel(const float* __restrict__ xc, const float* __restrict__ vc,
                                     const int* __restrict__ to_caller, float4* __restrict__ x, float4* __restrict__ x0,
                                     float4* __restrict__ vel, int n, int has_v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t o = 3 * (size_t)to_caller[i];
    const float m = x0[i].w;
    float4 p = make_float4(xc[o], xc[o + 1], xc[o + 2], m);
    x0[i] = p;
    x[i] = make_float4(p.x, p.y, p.z, 0.f);
    const float keep = vel[i].w;  // the bending diagonal stays
    vel[i] = has_v ? make_float4(vc[o], vc[o + 1], vc[o + 2], keep) : make_float4(0.f, 0.f, 0.f, keep);
}

__global__ void gather_state_kernel(const float4* __restrict__ src, const int* __restrict__ to_caller,
                                    float* __restrict__ dst, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t o = 3 * (size_t)to_caller[i];
    const float4 p = src[i];
    dst[o] = p.x;
    dst[o + 1] = p.y;
    dst[o + 2] = p.z;
}

__global__ void scatter_positions_kernel(const float* __restrict__ xc, const int* __restrict__ to_caller,
                                         float4* __restrict__ x, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t o = 3 * (size_t)to_caller[i];
    x[i] = make_float4(xc[o], xc[o + 1], xc[o + 2], 0.f);
}

// ---- FP64 reductions (deterministic: fixed element -> thread assignment, fixed tree)
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x 148 SMs

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] += sh[t + s];
        __syncthreads();
    }
    double r = sh[0];
    __syncthreads();
    return r;
}

struct EnergyArgs {
    const float4* x;
    const float4* x0;
    const float4* vel;
    const float4* vm;
    const float4* inst;
    int nv;
    const int2* edge;
    const float* rest;
    const float* kst;
    int ne;
    const int4* bend;
    const float* q16;
    const float* kb;
    int nb;
    double h;
    double* partial;  // 3 * gridDim.x
};

// Energy::compute_energy_inertia / _stretch_mass_spring / _bending
// (xpbd_constraints.h:2079-2214), every term in FP64.
__global__ void __launch_bounds__(kRedThreads) energy_kernel(EnergyArgs a) {
    __shared__ double sh[kRedThreads];
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double ei = 0.0, es = 0.0, eb = 0.0;
    for (int i = t0; i < a.nv; i += stride) {
        float4 p = a.x[i], q = a.x0[i], v = a.vel[i], mv = a.vm[i];
        float4 acc = a.inst[__float_as_int(mv.w)];
        bool pinned = mv.y != 0.f;
        double ax = pinned ? 0.0 : acc.x, ay = pinned ? 0.0 : acc.y, az = pinned ? 0.0 : acc.z;
        double dx = (double)p.x - ((double)q.x + a.h * v.x + a.h * a.h * ax);
        double dy = (double)p.y - ((double)q.y + a.h * v.y + a.h * a.h * ay);
        double dz = (double)p.z - ((double)q.z + a.h * v.z + a.h * a.h * az);
        ei += (double)q.w / (2.0 * a.h * a.h) * (dx * dx + dy * dy + dz * dz);
    }
    for (int i = t0; i < a.ne; i += stride) {
        int2 e = a.edge[i];
        float4 p0 = a.x[e.x], p1 = a.x[e.y];
        double dx = (double)p1.x - p0.x, dy = (double)p1.y - p0.y, dz = (double)p1.z - p0.z;
        double l2 = dx * dx + dy * dy + dz * dz;
        if (l2 < 1e-8) continue;
        double C = sqrt(l2) - (double)a.rest[i];
        es += 0.5 * (double)a.kst[i] * C * C;
    }
    for (int i = t0; i < a.nb; i += stride) {
        int4 id = a.bend[i];
        const int vid[4] = {id.x, id.y, id.z, id.w};
        double p[4][3];
        for (int j = 0; j < 4; ++j) {
            float4 t = a.x[vid[j]];
            p[j][0] = t.x;
            p[j][1] = t.y;
            p[j][2] = t.z;
        }
        const float* Q = a.q16 + 16 * (size_t)i;
        double s = 0.0;
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r)
                s += (double)Q[4 * c + r] * (p[c][0] * p[r][0] + p[c][1] * p[r][1] + p[c][2] * p[r][2]);
        eb += 0.5 * (double)a.kb[i] * s;
    }
    double si = block_sum(ei, sh);
    double ss = block_sum(es, sh);
    double sb = block_sum(eb, sh);
    if (threadIdx.x == 0) {
        a.partial[3 * blockIdx.x + 0] = si;
        a.partial[3 * blockIdx.x + 1] = ss;
        a.partial[3 * blockIdx.x + 2] = sb;
    }
}

__global__ void __launch_bounds__(kRedThreads) sum_partials3_kernel(const double* partial, int n, double* out) {
    __shared__ double sh[kRedThreads];
    for (int k = 0; k < 3; ++k) {
        double v = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[3 * i + k];
        double s = block_sum(v, sh);
        if (threadIdx.x == 0) out[k] = s;
    }
}

// Per-vertex FP64 evaluation of the incremental potential
//   G(z) = sum m/(2h^2)|z - y|^2 + sum 1/2 k (l - L)^2 + 1/2 sum_b k_b z^T Q_b z
// over the sliced-ELL stencil of the sweep, its rows loaded up front (all stencil
// entries, then all gathers) as in vbd_sweep_kernel:
//   kEvalGrad     out0[v] = |grad_v G(x)|^2 at free vertices (0 when pinned), with
//                 grad = m/h^2 (x - y) - f_stretch + sum_u W_vu (x_u - x_v),
//                 y = x0 + h v + h^2 a;
//   kEvalPot      out0[v] = the vertex's share of G(x): its inertia term against
//                 y = x0 + h v + h^2 a (a = 0 at pinned vertices, as
//                 Energy::compute_energy_inertia, xpbd_constraints.h:2079-2098), a
//                 quarter k (l - L)^2 per incident spring (each spring is seen from both
//                 ends) and -1/4 sum_u W_vu |x_u - x_v|^2, which sums to the bending
//                 energy because the merged stencil W is symmetric with zero row sums
//                 (x^T W x = -1/2 sum_{v,u} W_vu |x_u - x_v|^2);
//   kEvalPotPair  out0[v], out1[v] = the shares of G(x) and G(y) with y the saved
//                 inertial prediction (the inertia term of G(y) is 0).
// kEvalGradF32 (stencil_grad32_kernel) is kEvalGrad with the per-vertex gradient in
// the sweep's own FP32 arithmetic; only the sum over vertices is FP64.
constexpr int kEvalGrad = 0, kEvalPot = 1, kEvalPotPair = 2;
// Resident CTAs of `kernel` at `block` threads and `smem` bytes of dynamic shared
// memory, all SMs together (the grid of the kernels that stride over their work).
// A kernel with dynamic shared memory is allowed the device's whole opt-in amount, not
// just this block size's need: the resident counts are cached per block size, and an
// attribute sized for one block size would make a later launch at a larger one fail.
template <typename K>
int resident_ctas(K kernel, int block, size_t smem, int sms) {
    int res = 0;
    if (smem > 0) {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, kernel);
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             std::max((int)smem, optin - (int)fa.sharedSizeBytes));
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    }
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, kernel, block, smem);
    return std::max(1, sms) * (e == cudaSuccess && res > 0 ? res : 1);
}

struct EvalArgs {
    const float4* x;
    const float4* y;  // kEvalPotPair only
    const float4* x0;
    const float4* vel;
    const float4* vm;
    const float4* inst;
    const int2* st_iw;
    const float* st_rest;
    const int4* slices;
    const int* slice_inst;
    int nslices;
    double h;
    double* out0;
    double* out1;
    const int* active;  // per instance; null = all. Frozen instances keep their values.
};

template <int MODE>
__device__ __forceinline__ void eval_row(float4 xv, float4 xu, float4 yv, float4 yu, float L, float w, double ks,
                                         double& a0, double& a1, double& a2) {
    const double dx = (double)xu.x - xv.x, dy = (double)xu.y - xv.y, dz = (double)xu.z - xv.z;
    const double dd = dx * dx + dy * dy + dz * dz;
    if (MODE == kEvalGrad) {
        a0 += w * dx;
        a1 += w * dy;
        a2 += w * dz;
        if (L >= 0.f && dd > 0.0) {
            const double l = sqrt(dd);
            const double s = ks * (l - L) / l;
            a0 -= s * dx;
            a1 -= s * dy;
            a2 -= s * dz;
        }
    } else {
        a0 -= 0.25 * w * dd;
        if (L >= 0.f) {
            const double cx = sqrt(dd) - L;
            a0 += 0.25 * ks * cx * cx;
        }
        if (MODE == kEvalPotPair) {
            const double ex = (double)yu.x - yv.x, ey = (double)yu.y - yv.y, ez = (double)yu.z - yv.z;
            const double ee = ex * ex + ey * ey + ez * ez;
            a1 -= 0.25 * w * ee;
            if (L >= 0.f) {
                const double cy = sqrt(ee) - L;
                a1 += 0.25 * ks * cy * cy;
            }
        }
    }
}

// One slice of an FP64 stencil pass; the data read once per pass (stencil rows, vertex
// records, frame-start state) through evict-first loads.
template <int TPV, int RE, int RB, int MODE>
__device__ __forceinline__ void eval_slice(const EvalArgs& a, int slice, int lane) {
    const int4 sd = __ldg(&a.slices[slice]);
    const int rows = sd.w & 0xffff, erows = sd.w >> 16, brows = rows - erows;
    const int k = lane / TPV;
    const bool leader = k < sd.y && (lane % TPV) == 0;
    const int v = sd.x + min(k, sd.y - 1);
    const int base = sd.z + lane;
    const int bbase = base + erows * 32;
    const float4 mv = __ldcs(&a.vm[v]);
    int ue[RE], ub[RB];
    float we[RE], le[RE], wb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) {
        ue[r] = v;
        we[r] = 0.f;
        le[r] = -1.f;
        if (r < erows) {
            const int2 iw = __ldcs(&a.st_iw[base + r * 32]);
            ue[r] = iw.x;
            we[r] = __int_as_float(iw.y);
            le[r] = __ldcs(&a.st_rest[base + r * 32]);
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        ub[r] = v;
        wb[r] = 0.f;
        if (r < brows) {
            const int2 iw = __ldcs(&a.st_iw[bbase + r * 32]);
            ub[r] = iw.x;
            wb[r] = __int_as_float(iw.y);
        }
    }
    const float4 ip = __ldg(&a.inst[__float_as_int(mv.w)]);
    const double ks = ip.w;
    const float4 xv = a.x[v];
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 yv = MODE == kEvalPotPair ? a.y[v] : zero;
    float4 xe[RE], xb[RB], ye[RE], yb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) {
        xe[r] = a.x[ue[r]];
        ye[r] = MODE == kEvalPotPair ? a.y[ue[r]] : zero;
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        xb[r] = a.x[ub[r]];
        yb[r] = MODE == kEvalPotPair ? a.y[ub[r]] : zero;
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int r = 0; r < RE; ++r) eval_row<MODE>(xv, xe[r], yv, ye[r], le[r], we[r], ks, a0, a1, a2);
    for (int r = RE; r < erows; ++r) {
        const int2 iw = __ldg(&a.st_iw[base + r * 32]);
        eval_row<MODE>(xv, a.x[iw.x], yv, MODE == kEvalPotPair ? a.y[iw.x] : zero, __ldg(&a.st_rest[base + r * 32]),
                       __int_as_float(iw.y), ks, a0, a1, a2);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) eval_row<MODE>(xv, xb[r], yv, yb[r], -1.f, wb[r], ks, a0, a1, a2);
    for (int r = RB; r < brows; ++r) {
        const int2 iw = __ldg(&a.st_iw[bbase + r * 32]);
        eval_row<MODE>(xv, a.x[iw.x], yv, MODE == kEvalPotPair ? a.y[iw.x] : zero, -1.f, __int_as_float(iw.y), ks, a0,
                       a1, a2);
    }
#pragma unroll
    for (int o = TPV / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (!leader) return;
    const float4 p0 = __ldcs(&a.x0[v]);
    const double h = a.h, m = p0.w;
    if (MODE == kEvalGrad) {
        if (mv.y != 0.f) {
            a.out0[v] = 0.0;
            return;
        }
        const float4 vv = __ldcs(&a.vel[v]);
        a0 += m / (h * h) * ((double)xv.x - ((double)p0.x + h * vv.x + h * h * ip.x));
        a1 += m / (h * h) * ((double)xv.y - ((double)p0.y + h * vv.y + h * h * ip.y));
        a2 += m / (h * h) * ((double)xv.z - ((double)p0.z + h * vv.z + h * h * ip.z));
        a.out0[v] = a0 * a0 + a1 * a1 + a2 * a2;
    } else if (MODE == kEvalPot) {
        const float4 vv = __ldcs(&a.vel[v]);
        const bool pinned = mv.y != 0.f;
        const double ax = pinned ? 0.0 : ip.x, ay = pinned ? 0.0 : ip.y, az = pinned ? 0.0 : ip.z;
        const double dx = (double)xv.x - ((double)p0.x + h * vv.x + h * h * ax);
        const double dy = (double)xv.y - ((double)p0.y + h * vv.y + h * h * ay);
        const double dz = (double)xv.z - ((double)p0.z + h * vv.z + h * h * az);
        a.out0[v] = a0 + m / (2.0 * h * h) * (dx * dx + dy * dy + dz * dz);
    } else {
        const double dx = (double)xv.x - yv.x, dy = (double)xv.y - yv.y, dz = (double)xv.z - yv.z;
        a.out0[v] = a0 + m / (2.0 * h * h) * (dx * dx + dy * dy + dz * dz);
        a.out1[v] = a1;
    }
}

// An FP64 stencil pass over a resident grid, slices taken as in stencil_grad32_kernel:
// warp w takes slices w, w + nwarps, ..., and runs those of active instances only.
template <int TPV, int RE, int RB, int MODE>
__global__ void __launch_bounds__(128) stencil_eval_kernel(EvalArgs a) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    for (int round = w; round < a.nslices; round += 32 * nwarps) {
        const int s = round + lane * nwarps;
        const bool want = s < a.nslices && (!a.active || a.active[__ldg(&a.slice_inst[s])]);
        unsigned m = __ballot_sync(0xffffffffu, want);
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            eval_slice<TPV, RE, RB, MODE>(a, round + j * nwarps, lane);
        }
    }
}

// Resident CTAs of stencil_eval_kernel<..., MODE>, all SMs (queried on first use).
template <int TPV, int RE, int RB, int MODE>
int eval_ctas() {
    static int n = 0;
    if (!n) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        n = resident_ctas(stencil_eval_kernel<TPV, RE, RB, MODE>, 128, 0, sms);
    }
    return n;
}

template <int MODE>
cudaError_t stencil_eval_launch(int tpv, const EvalArgs& a, cudaStream_t st) {
    const int blocks = (a.nslices * 32 + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    switch (tpv) {
        case 1: stencil_eval_kernel<1, 6, 6, MODE><<<std::min(blocks, eval_ctas<1, 6, 6, MODE>()), 128, 0, st>>>(a); break;
        case 2: stencil_eval_kernel<2, 3, 3, MODE><<<std::min(blocks, eval_ctas<2, 3, 3, MODE>()), 128, 0, st>>>(a); break;
        case 4: stencil_eval_kernel<4, 2, 2, MODE><<<std::min(blocks, eval_ctas<4, 2, 2, MODE>()), 128, 0, st>>>(a); break;
        default: stencil_eval_kernel<8, 1, 1, MODE><<<std::min(blocks, eval_ctas<8, 1, 1, MODE>()), 128, 0, st>>>(a); break;
    }
    count_launch(st);
    return cudaGetLastError();
}

// Deterministic per-instance sum of g2 over the instance's layout range, two levels:
// block (chunk j, instance i) sums a fixed strided subset, then one block per
// instance adds the kSegChunks partials in order.
constexpr int kSegChunks = 32;
__global__ void __launch_bounds__(kRedThreads) segment_partial_kernel(const double* g2, const int* seg, double* partial,
                                                                      const int* mask) {
    __shared__ double sh[kRedThreads];
    const int i = blockIdx.y, j = blockIdx.x;
    if (mask && !mask[i]) return;  // block-uniform: the instance keeps its previous value
    const int b = seg[i], e = seg[i + 1];
    double v = 0.0;
    for (int t = b + j * kRedThreads + threadIdx.x; t < e; t += kSegChunks * kRedThreads) v += g2[t];
    double s = block_sum(v, sh);
    if (threadIdx.x == 0) partial[i * kSegChunks + j] = s;
}

__global__ void __launch_bounds__(kSegChunks) segment_final_kernel(const double* partial, double* out, int take_sqrt,
                                                                   const int* mask) {
    __shared__ double sh[kSegChunks];
    if (mask && !mask[blockIdx.x]) return;
    double s = block_sum(partial[blockIdx.x * kSegChunks + threadIdx.x], sh);
    if (threadIdx.x == 0) out[blockIdx.x] = take_sqrt ? sqrt(s) : s;
}

// Bookkeeping of the residual-driven frame (one block). The probe schedule lives on the
// device, so that the same captured chunk graph serves every probe point: pts[0..n-1]
// are the iteration counts at which probes may run and pts[n] = max_iters; *pidx is the
// index of the probe point just reached (advanced here, once per call).
// init: norm0 = ||grad G(y)||, every instance with a nonzero gradient active, *pidx = 0.
// Otherwise, after done = pts[*pidx] iterations: every active instance has iters = done;
// an instance probed now (due) stops when ||grad G|| <= tols[i] ||grad G(y)|| or
// done >= max_iters. Then due is set for the next point `next`, by the probe policy:
//   0 (fixed)        next == max_iters, or next >= first[i] and (next - first[i]) a
//                    multiple of step;
//   1 (extrapolated) next == max_iters, or next >= next_due[i]. After the first probe
//                    next_due = that point + step; after later ones the contraction per
//                    iteration since the previous probe, rho, predicts the iterations
//                    still needed, log(tol / r) / log(rho), and the next probe comes after
//                    half of them (at least step, rounded up to a multiple of it); without
//                    progress (rho >= 1) it comes at the cap. A flat residual curve is
//                    then probed a few times per frame instead of every step.
__global__ void __launch_bounds__(256) residual_check_kernel(const double* norm, double* norm0, int* active, int* iters,
                                                            int* n_active, int* due, int ninst, int init,
                                                            const int* pts, int* pidx, int step, const int* first,
                                                            int max_iters, const double* tols, int policy,
                                                            int* next_due, int* last_it, double* last_res) {
    __shared__ int count[256];
    const int p = init ? 0 : *pidx;
    const int done = init ? 0 : pts[p];
    const int next = init ? pts[0] : pts[p + 1];
    int c = 0;
    for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
        if (init) {
            norm0[i] = norm[i];
            active[i] = norm[i] > 0.0 && max_iters > 0 ? 1 : 0;
            iters[i] = 0;
            next_due[i] = first[i];
            last_it[i] = 0;
            last_res[i] = 1.0;
        } else if (active[i]) {
            iters[i] = done;
            if (due[i]) {
                const double r = norm0[i] > 0.0 ? norm[i] / norm0[i] : 0.0;
                if (norm[i] <= tols[i] * norm0[i] || done >= max_iters) {
                    active[i] = 0;
                } else if (policy == 1) {
                    int gap = step;
                    if (last_it[i] > 0) {
                        gap = max_iters - done;
                        if (r < last_res[i] && r > 0.0 && tols[i] > 0.0) {
                            const double rho = pow(r / last_res[i], 1.0 / (double)(done - last_it[i]));
                            const double need = log(tols[i] / r) / log(rho);  // > 0: r > tol, rho < 1
                            if (need < (double)(max_iters - done)) {
                                const int half = (int)ceil(0.5 * need);
                                gap = ((max(half, step) + step - 1) / step) * step;
                            }
                        }
                    }
                    next_due[i] = min(done + gap, max_iters);
                    last_it[i] = done;
                    last_res[i] = r;
                }
            }
        }
        const int f = first[i];
        const bool sched = policy == 1 ? next >= next_due[i] : (next >= f && (next - f) % step == 0);
        due[i] = active[i] && (next >= max_iters || sched) ? 1 : 0;
        c += active[i];
    }
    count[threadIdx.x] = c;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) count[threadIdx.x] += count[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *n_active = count[0];
        *pidx = init ? 0 : p + 1;
    }
}

// Self-test of the bounded waits (ats_selftest_bounded_waits): each kernel waits for
// something that never happens and must give up after `polls` polls with its error
// word set. One block waits at a grid barrier for twice the blocks launched; one block
// waits on an mbarrier on which nothing arrives.
__global__ void selftest_barrier_kernel(unsigned* bar, int* err, unsigned polls) {
    unsigned target = gridDim.x;  // grid_barrier adds gridDim.x: 2 x the arrivals there will be
    grid_barrier(bar, err, target, polls);
}

__global__ void selftest_mbarrier_kernel(int* err, unsigned polls) {
    __shared__ __align__(8) uint64_t mbar;
    if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
    __syncthreads();
    const bool ok = umma::mbar_wait(&mbar, 0, polls);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    __syncthreads();
}

__global__ void selftest_touch_kernel(int* out) {
    if (threadIdx.x == 0) *out = 12345;
}

}  // namespace
}  // namespace ats

using namespace ats;

namespace ats {

template <typename T, typename U>
int upload(DevBuf<T>& d, const std::vector<U>& h, size_t count) {
    if (d.p) {
        cudaFree(d.p);
        d.p = nullptr;
    }
    ATS_CUDA(d.alloc(count));
    if (count) ATS_CUDA(cudaMemcpy(d.p, h.data(), count * sizeof(T), cudaMemcpyHostToDevice));
    return ATS_OK;
}

int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(std::string("no CUDA device: ") + (e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e)));
        return ATS_ERR_CUDA;
    }
    return ATS_OK;
}

int upload_stencil(ats_cloth* c) {
    int r;
    const Layout& L = c->L;
    if ((r = upload(c->st_iw, L.st_iw, L.st_rest.size())) || (r = upload(c->st_rest, L.st_rest, L.st_rest.size())) ||
        (r = upload(c->slices, L.slices, L.slices.size() / 4)))
        return r;
    // a slice lies in one instance: the instance id of its first vertex
    std::vector<int> si(L.slices.size() / 4);
    for (size_t k = 0; k < si.size(); ++k) std::memcpy(&si[k], &L.vm[4 * (size_t)L.slices[4 * k] + 3], sizeof(int));
    // and its pinned vertices (bit k: vertex vbegin + k), for the sweeps that skip vm
    std::vector<int2> sm(si.size());
    for (size_t k = 0; k < si.size(); ++k) {
        unsigned pins = 0;
        const int vb = L.slices[4 * k], nvs = L.slices[4 * k + 1];
        for (int j = 0; j < nvs && j < 32; ++j)
            if (L.vm[4 * (size_t)(vb + j) + 1] != 0.f) pins |= 1u << j;
        sm[k] = make_int2(si[k], (int)pins);
    }
    if ((r = upload(c->slice_inst, si, si.size())) || (r = upload(c->slice_meta, sm, sm.size())) ||
        (r = upload(c->color_slices, L.color_slices, L.color_slices.size())))
        return r;
    // per-colour lists of the slices still iterating (residual-driven frames)
    std::vector<int> zeros(std::max<size_t>(si.size(), 1), 0);
    if ((r = upload(c->act_list, zeros, si.size())) ||
        (r = upload(c->act_count, zeros, std::max(1, L.n_vcolors))))
        return r;
    return ATS_OK;
}

// The slices of instances still active, listed per colour at the colour's slice
// offset (a warp appends its run of one colour with one atomic). counts must be zero.
__global__ void compact_slices_kernel(const int* __restrict__ slice_inst, const int* __restrict__ active,
                                      const int* __restrict__ color_begin, int ncolors, int nslices,
                                      int* __restrict__ list, int* __restrict__ counts) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int col = -1;
    bool act = false;
    if (s < nslices) {
        act = active[slice_inst[s]] != 0;
        col = 0;
        while (col + 1 < ncolors && s >= color_begin[col + 1]) ++col;
    }
    const unsigned actm = __ballot_sync(0xffffffffu, act);
    const unsigned peers = __match_any_sync(0xffffffffu, col) & actm;
    const int leader = peers ? __ffs(peers) - 1 : lane;
    int base = 0;
    if (act && lane == leader) base = atomicAdd(&counts[col], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (act) list[color_begin[col] + base + __popc(peers & ((1u << lane) - 1u))] = s;
}

int enqueue_compaction(ats_cloth* c, cudaStream_t st) {
    const int n = (int)c->slices.n, nc = c->L.n_vcolors;
    if (n == 0 || nc == 0) return ATS_OK;
    ATS_CUDA(cudaMemsetAsync(c->act_count.p, 0, nc * sizeof(int), st));
    compact_slices_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->slice_inst.p, c->active.p, c->color_slices.p, nc, n,
                                                           c->act_list.p, c->act_count.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    return ATS_OK;
}

// Dynamic shared memory of vbd_sweep_pipe_kernel: two slice stages per warp.
template <int RE, int RB>
constexpr size_t pipe_smem_per_warp() {
    return 2 * sizeof(SliceStage<RE, RB>);
}

// Resident CTAs of the list sweeps (form 0: vbd_sweep_list_kernel, 1:
// vbd_sweep_pipe_kernel, 2: vbd_sweep_stream_kernel), all SMs together, per (lanes per
// vertex, block size); queried (and the pipelined kernel's shared-memory attributes
// set) on first use, which is
// outside stream capture (the eager iterations of ats_frame_to_residual's first frame,
// or ats_autotune, come first).
template <int TPV, int RE, int RB>
int list_form_ctas(int form, int block, int sms) {
    switch (form) {
        case 1: return resident_ctas(vbd_sweep_pipe_kernel<TPV, RE, RB>, block, (block / 32) * pipe_smem_per_warp<RE, RB>(), sms);
        case 2: return resident_ctas(vbd_sweep_stream_kernel<TPV, RE, RB>, block, 0, sms);
        default: return resident_ctas(vbd_sweep_list_kernel<TPV, RE, RB>, block, 0, sms);
    }
}
int list_sweep_ctas(int tpv, int block, int form) {
    static int cache[3][4][3] = {};
    const int ti = tpv == 1 ? 0 : tpv == 2 ? 1 : tpv == 4 ? 2 : 3, bi = block == 64 ? 0 : block == 128 ? 1 : 2;
    int& slot = cache[form >= 0 && form < 3 ? form : 0][ti][bi];
    if (!slot) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        switch (tpv) {
            case 1: slot = list_form_ctas<1, 6, 6>(form, block, sms); break;
            case 2: slot = list_form_ctas<2, 3, 3>(form, block, sms); break;
            case 4: slot = list_form_ctas<4, 2, 2>(form, block, sms); break;
            default: slot = list_form_ctas<8, 1, 1>(form, block, sms); break;
        }
    }
    return slot;
}

// listed: 0 one-wave sweep over the colour's slices, 1 list sweep, 2 pipelined list
// sweep, 3 streamed list sweep; a list sweep given a window `win` carries it as its
// access-policy window (positions as persisting L2 lines)
template <int TPV, int RE, int RB>
cudaError_t sweep_launch(dim3 grid, dim3 block, cudaStream_t st, const SweepArgs& a, int listed,
                         const cudaAccessPolicyWindow* win = nullptr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = listed == 2 ? (block.x / 32) * pipe_smem_per_warp<RE, RB>() : 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (listed > 0 && win && win->num_bytes > 0) {
        attr[1].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[1].val.accessPolicyWindow = *win;
        cfg.numAttrs = 2;
    }
    const cudaError_t e = listed == 3   ? cudaLaunchKernelEx(&cfg, vbd_sweep_stream_kernel<TPV, RE, RB>, a)
                          : listed == 2 ? cudaLaunchKernelEx(&cfg, vbd_sweep_pipe_kernel<TPV, RE, RB>, a)
                          : listed == 1 ? cudaLaunchKernelEx(&cfg, vbd_sweep_list_kernel<TPV, RE, RB>, a)
                                        : cudaLaunchKernelEx(&cfg, vbd_sweep_kernel<TPV, RE, RB>, a);
    if (e == cudaSuccess) count_launch(st);
    return e;
}

// Persisting positions keep a handle's positions in L2 between colours: a list sweep
// streams about three times the positions' bytes of stencil past them, and the next
// colours gather them again as neighbours. The handles that use it share the context's persisting-L2
// set-aside (cudaLimitPersistingL2CacheSize, a per-context limit): the first one sizes
// it for its positions (up to the device maximum), the last one puts back the size it
// found and resets the persisting lines. Each launch of its sweep carries an access-policy
// window over the handle's positions whose hit ratio is the set-aside over the window.
// Per device: the handles holding a share and the set-aside size found before the first.
struct L2Share {
    int users = 0;
    size_t prev = 0;
};
std::mutex g_l2_mu;
std::map<int, L2Share> g_l2;

// Makes `dev` current for the scope (the limit calls act on the current device).
struct CurrentDevice {
    int prev = -1;
    explicit CurrentDevice(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~CurrentDevice() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

int l2_keep_acquire(ats_cloth* c) {
    if (c->l2_keep) return ATS_OK;
    CurrentDevice on(c->device);
    int max_persist = 0, max_window = 0;
    ATS_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, c->device));
    ATS_CUDA(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, c->device));
    if (max_persist <= 0 || max_window <= 0) {
        set_error("persisting positions: the device has no persisting L2");
        return ATS_ERR_STATE;
    }
    const size_t window = std::min(c->x.bytes(), (size_t)max_window);
    size_t setaside = 0;
    {
        std::lock_guard<std::mutex> lk(g_l2_mu);
        L2Share& sh = g_l2[c->device];
        size_t cur = 0;
        ATS_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
        const size_t want = std::min(window, (size_t)max_persist);
        if (want > cur) ATS_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
        ATS_CUDA(cudaDeviceGetLimit(&setaside, cudaLimitPersistingL2CacheSize));
        if (sh.users++ == 0) sh.prev = cur;
    }
    c->l2_window.base_ptr = c->x.p;
    c->l2_window.num_bytes = window;
    c->l2_window.hitRatio = window > 0 ? std::min(1.f, (float)((double)setaside / (double)window)) : 0.f;
    c->l2_window.hitProp = cudaAccessPropertyPersisting;
    c->l2_window.missProp = cudaAccessPropertyNormal;
    c->l2_keep = true;
    return ATS_OK;
}

void l2_keep_release(ats_cloth* c) {
    if (!c->l2_keep) return;
    c->l2_keep = false;
    c->l2_window = cudaAccessPolicyWindow{};
    CurrentDevice on(c->device);
    std::lock_guard<std::mutex> lk(g_l2_mu);
    L2Share& sh = g_l2[c->device];
    if (--sh.users == 0) {
        cudaDeviceSynchronize();
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, sh.prev);
    }
}

// Sets the list form of a handle (resident grid queried outside any capture).
int set_list_form(ats_cloth* c, int form) {
    c->list_form = form;
    list_sweep_ctas(c->L.tpv, c->block, form);
    return ATS_OK;
}

// Takes or gives back the handle's share of the persisting-L2 set-aside.
int set_l2_persisting(ats_cloth* c, bool on) {
    if (on) return l2_keep_acquire(c);
    l2_keep_release(c);
    return ATS_OK;
}

int launch_sweep(ats_cloth* c, int color, cudaStream_t st, const int* active) {
    const int sb = c->L.color_slices[color], se = c->L.color_slices[color + 1];
    if (se <= sb) return ATS_OK;
    SweepArgs a;
    a.x = c->x.p;
    a.x0 = c->x0.p;
    a.vel = c->vel.p;
    a.vm = c->vm.p;
    a.st_iw = c->st_iw.p;
    a.st_rest = c->st_rest.p;
    a.slices = c->slices.p;
    a.slice_inst = c->slice_inst.p;
    a.slice_meta = c->slice_meta.p;
    a.inst = c->inst.p;
    // with an activity mask: only the slices the last compaction listed (the mask
    // itself is what the compaction read)
    const int listed = active != nullptr ? 1 + c->list_form : 0;
    a.active = nullptr;  // masked sweeps go through the lists
    a.list = listed ? c->act_list.p + sb : nullptr;
    a.list_count = listed ? c->act_count.p + color : nullptr;
    a.slice_begin = sb;
    a.slice_end = se;
    a.h = c->h;
    a.h2inv = c->h2inv;
    const int warps_per_block = c->block / 32;
    int blocks = (se - sb + warps_per_block - 1) / warps_per_block;
    if (listed) blocks = std::min(blocks, list_sweep_ctas(c->L.tpv, c->block, c->list_form));
    const dim3 grid(blocks), block(c->block);
    cudaError_t e;
    switch (c->L.tpv) {
        case 1: e = sweep_launch<1, 6, 6>(grid, block, st, a, listed, &c->l2_window); break;
        case 2: e = sweep_launch<2, 3, 3>(grid, block, st, a, listed, &c->l2_window); break;
        case 4: e = sweep_launch<4, 2, 2>(grid, block, st, a, listed, &c->l2_window); break;
        default: e = sweep_launch<8, 1, 1>(grid, block, st, a, listed, &c->l2_window); break;
    }
    if (e != cudaSuccess) {
        set_error(std::string("vbd sweep launch: ") + cudaGetErrorString(e));
        return ATS_ERR_CUDA;
    }
    return ATS_OK;
}

int launch_predict(ats_cloth* c, cudaStream_t st) {
    const int n = c->L.nv;
    predict_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->x.p, c->x0.p, c->vel.p, c->vm.p, c->inst.p, n, c->h); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    return ATS_OK;
}

int launch_update(ats_cloth* c, cudaStream_t st) {
    const int n = c->L.nv;
    update_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->x.p, c->x0.p, c->vel.p, n, c->h, c->damp); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    return ATS_OK;
}

int launch_reset(ats_cloth* c, cudaStream_t st) {
    if (c->xs_lambda.n) ATS_CUDA(cudaMemsetAsync(c->xs_lambda.p, 0, c->xs_lambda.bytes(), st));
    if (c->xb_lambda.n) ATS_CUDA(cudaMemsetAsync(c->xb_lambda.p, 0, c->xb_lambda.bytes(), st));
    return ATS_OK;
}

// a launch that may begin while the previous kernel of the stream drains
// (programmatic dependent launch; the kernel waits with griddepcontrol.wait)
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), int blocks, int threads, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args...);
    if (e == cudaSuccess) count_launch(st);
    return e;
}

int launch_xpbd_stretch(ats_cloth* c, int color, cudaStream_t st) {
    const int b = c->L.xs_color[color], e = c->L.xs_color[color + 1];
    if (e <= b) return ATS_OK;
    ATS_CUDA(launch_pdl(xpbd_stretch_kernel, (e - b + 127) / 128, 128, st, c->x.p, (const float4*)c->vm.p,
                        (const int2*)c->xs_edge.p, (const float*)c->xs_rest.p, (const float*)c->xs_k.p,
                        c->xs_lambda.p, b, e, c->h));
    return ATS_OK;
}

int launch_xpbd_bending(ats_cloth* c, int color, cudaStream_t st) {
    const int b = c->L.xb_color[color], e = c->L.xb_color[color + 1];
    if (e <= b) return ATS_OK;
    ATS_CUDA(launch_pdl(xpbd_bending_kernel, (e - b + 127) / 128, 128, st, c->x.p, (const float4*)c->vm.p,
                        (const int4*)c->xb_idx.p, (const float4*)c->xb_q.p, c->xb_lambda.p, b, e, c->h));
    return ATS_OK;
}

// `iterations` XPBD iterations as one cooperative launch of xpbd_loop_kernel (one
// block per SM), the barrier state reset on the stream first.
int launch_xpbd_loop_once(ats_cloth* c, const XpbdLoopArgs& a, cudaStream_t st);

int launch_xpbd_loop(ats_cloth* c, int iterations, cudaStream_t st) {
    XpbdLoopArgs a;
    a.x = c->x.p;
    a.vm = c->vm.p;
    a.edge = (const int2*)c->xs_edge.p;
    a.rest = c->xs_rest.p;
    a.kst = c->xs_k.p;
    a.slambda = c->xs_lambda.p;
    a.bidx = (const int4*)c->xb_idx.p;
    a.bq = (const float4*)c->xb_q.p;
    a.blambda = c->xb_lambda.p;
    a.scolor = c->xs_color_d.p;
    a.bcolor = c->xb_color_d.p;
    a.nsc = c->L.n_scolors;
    a.nbc = c->L.n_bcolors;
    a.h = c->h;
    a.bar = c->loop_bar.p;
    a.err = c->loop_err.p;
    // at most kMaxLoopArrivals barrier arrivals per launch
    const unsigned long long per_it =
        std::max(1ull, (unsigned long long)(a.nsc + a.nbc) * (unsigned long long)c->xpbd_loop_blocks);
    const int max_it = (int)std::min<unsigned long long>(kMaxLoopArrivals / per_it, 1ull << 30);
    if (max_it < 1) {
        set_error("xpbd loop: too many colours x blocks for one launch");
        return ATS_ERR_INVALID;
    }
    for (int done = 0; done < iterations;) {
        a.iterations = std::min(iterations - done, max_it);
        done += a.iterations;
        const int r = launch_xpbd_loop_once(c, a, st);
        if (r) return r;
    }
    return ATS_OK;
}

int launch_xpbd_loop_once(ats_cloth* c, const XpbdLoopArgs& a, cudaStream_t st) {
    ATS_CUDA(cudaMemsetAsync(c->loop_bar.p, 0, 2 * sizeof(unsigned), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->xpbd_loop_blocks);
    cfg.blockDim = dim3(kXpbdLoopThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ATS_CUDA(cudaLaunchKernelEx(&cfg, xpbd_loop_kernel, a));
    count_launch(st);
    return ATS_OK;
}

// Co-resident blocks of vbd_loop_kernel at (lanes per vertex, block size), all SMs,
// queried outside any capture (at autotune time); 0 when cooperative launch is
// unavailable.
int vbd_loop_blocks(int tpv, int block, int device) {
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e;
    switch (tpv) {
        case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vbd_loop_kernel<1, 6, 6>, block, 0); break;
        case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vbd_loop_kernel<2, 3, 3>, block, 0); break;
        case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vbd_loop_kernel<4, 2, 2>, block, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vbd_loop_kernel<8, 1, 1>, block, 0); break;
    }
    return coop && e == cudaSuccess && per_sm > 0 ? sms * per_sm : 0;
}

int launch_vbd_loop_once(ats_cloth* c, const SweepArgs& a, const int* cs, int nc, int iterations, cudaStream_t st);

int launch_vbd_loop(ats_cloth* c, int iterations, cudaStream_t st) {
    SweepArgs a;
    a.x = c->x.p;
    a.x0 = c->x0.p;
    a.vel = c->vel.p;
    a.vm = c->vm.p;
    a.st_iw = c->st_iw.p;
    a.st_rest = c->st_rest.p;
    a.slices = c->slices.p;
    a.slice_inst = c->slice_inst.p;
    a.slice_meta = c->slice_meta.p;
    a.inst = c->inst.p;
    a.active = nullptr;
    a.list = nullptr;
    a.list_count = nullptr;
    a.slice_begin = 0;
    a.slice_end = (int)c->slices.n;
    a.h = c->h;
    a.h2inv = c->h2inv;
    const int* cs = c->color_slices.p;
    const int nc = c->L.n_vcolors;
    // at most kMaxLoopArrivals barrier arrivals per launch
    const unsigned long long per_it = std::max(1ull, (unsigned long long)nc * (unsigned long long)c->vbd_loop_blocks);
    const int max_it = (int)std::min<unsigned long long>(kMaxLoopArrivals / per_it, 1ull << 30);
    if (max_it < 1) {
        set_error("vbd loop: too many colours x blocks for one launch");
        return ATS_ERR_INVALID;
    }
    for (int done = 0; done < iterations;) {
        const int n = std::min(iterations - done, max_it);
        done += n;
        const int r = launch_vbd_loop_once(c, a, cs, nc, n, st);
        if (r) return r;
    }
    return ATS_OK;
}

int launch_vbd_loop_once(ats_cloth* c, const SweepArgs& a, const int* cs, int nc, int iterations, cudaStream_t st) {
    ATS_CUDA(cudaMemsetAsync(c->loop_bar.p, 0, 2 * sizeof(unsigned), st));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->vbd_loop_blocks);
    cfg.blockDim = dim3(c->block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    switch (c->L.tpv) {
        case 1: e = cudaLaunchKernelEx(&cfg, vbd_loop_kernel<1, 6, 6>, a, cs, nc, iterations, c->loop_bar.p, c->loop_err.p); break;
        case 2: e = cudaLaunchKernelEx(&cfg, vbd_loop_kernel<2, 3, 3>, a, cs, nc, iterations, c->loop_bar.p, c->loop_err.p); break;
        case 4: e = cudaLaunchKernelEx(&cfg, vbd_loop_kernel<4, 2, 2>, a, cs, nc, iterations, c->loop_bar.p, c->loop_err.p); break;
        default: e = cudaLaunchKernelEx(&cfg, vbd_loop_kernel<8, 1, 1>, a, cs, nc, iterations, c->loop_bar.p, c->loop_err.p); break;
    }
    if (e != cudaSuccess) {
        set_error(std::string("vbd loop launch: ") + cudaGetErrorString(e));
        return ATS_ERR_CUDA;
    }
    count_launch(st);
    return ATS_OK;
}

int enqueue_iterations(ats_cloth* c, int solver, int iterations, cudaStream_t st, const int* active) {
    int r;
    if (solver == ATS_SOLVER_VBD && !active && c->vbd_loop_blocks > 0 && iterations > 0 && c->L.n_vcolors > 0)
        return launch_vbd_loop(c, iterations, st);
    if (solver == ATS_SOLVER_XPBD && c->xpbd_loop_blocks > 0 && iterations > 0 &&
        c->L.n_scolors + c->L.n_bcolors > 0)
        return launch_xpbd_loop(c, iterations, st);
    for (int it = 0; it < iterations; ++it) {
        if (solver == ATS_SOLVER_VBD) {
            for (int col = 0; col < c->L.n_vcolors; ++col)
                if ((r = launch_sweep(c, col, st, active))) return r;
        } else {
            for (int col = 0; col < c->L.n_scolors; ++col)
                if ((r = launch_xpbd_stretch(c, col, st))) return r;
            for (int col = 0; col < c->L.n_bcolors; ++col)
                if ((r = launch_xpbd_bending(c, col, st))) return r;
        }
    }
    return ATS_OK;
}

int enqueue_frame(ats_cloth* c, int solver, cudaStream_t st) {
    int r;
    for (int sub = 0; sub < c->prm.num_substep; ++sub) {
        if ((r = launch_predict(c, st))) return r;
        if (solver == ATS_SOLVER_XPBD && (r = launch_reset(c, st))) return r;
        if ((r = enqueue_iterations(c, solver, c->prm.iterations, st))) return r;
        if ((r = launch_update(c, st))) return r;
    }
    return ATS_OK;
}

EvalArgs eval_args(ats_cloth* c) {
    EvalArgs a;
    a.x = c->x.p;
    a.y = nullptr;
    a.x0 = c->x0.p;
    a.vel = c->vel.p;
    a.vm = c->vm.p;
    a.inst = c->inst.p;
    a.st_iw = c->st_iw.p;
    a.st_rest = c->st_rest.p;
    a.slices = c->slices.p;
    a.slice_inst = c->slice_inst.p;
    a.nslices = (int)c->slices.n;
    a.h = (double)c->h;
    a.out0 = a.out1 = nullptr;
    a.active = nullptr;
    return a;
}

int segment_sum(ats_cloth* c, const double* per_vertex, double* out, int take_sqrt, cudaStream_t st,
                const int* mask = nullptr) {
    segment_partial_kernel<<<dim3(kSegChunks, c->L.ninst), kRedThreads, 0, st>>>(per_vertex, c->inst_seg.p,
                                                                                   c->seg_partial.p, mask); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    segment_final_kernel<<<c->L.ninst, kSegChunks, 0, st>>>(c->seg_partial.p, out, take_sqrt, mask); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    return ATS_OK;
}

// |grad_v G(x)|^2 per free vertex with the sweep's FP32 force arithmetic (vbd_edge,
// vbd_bend and the inertia term of vbd_sweep_kernel: grad = -f); only the squared norm
// and the sums over vertices are FP64. Used by the residual-driven frames, whose
// probes run every few iterations: the gradient terms of a vertex are far from
// cancelling at the residuals those frames stop at, so FP32 terms (as the reference
// energy's) lose nothing there, and this kernel needs half the registers of the FP64
// one.
// One slice; the data read once per probe (stencil rows, vertex records, frame-start
// state) through evict-first loads.
template <int TPV, int RE, int RB>
__device__ __forceinline__ void grad32_slice(const EvalArgs& a, int slice, int lane, float h, float h2inv) {
    const int4 sd = __ldg(&a.slices[slice]);
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
            const int2 iw = __ldcs(&a.st_iw[base + r * 32]);
            ue[r] = iw.x;
            we[r] = __int_as_float(iw.y);
            le[r] = __ldcs(&a.st_rest[base + r * 32]);
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        ub[r] = v;
        wb[r] = 0.f;
        if (r < brows) {
            const int2 iw = __ldcs(&a.st_iw[bbase + r * 32]);
            ub[r] = iw.x;
            wb[r] = __int_as_float(iw.y);
        }
    }
    const float4 mv = __ldcs(&a.vm[v]);
    const float4 ip = __ldg(&a.inst[__float_as_int(mv.w)]);
    const float4 xv = a.x[v];
    float4 xe[RE], xb[RB];
#pragma unroll
    for (int r = 0; r < RE; ++r) xe[r] = a.x[ue[r]];
#pragma unroll
    for (int r = 0; r < RB; ++r) xb[r] = a.x[ub[r]];
    float fx = 0.f, fy = 0.f, fz = 0.f, h00 = 0.f, h01 = 0.f, h02 = 0.f, h11 = 0.f, h12 = 0.f, h22 = 0.f;
#pragma unroll
    for (int r = 0; r < RE; ++r) vbd_edge(xv, xe[r], le[r], we[r], ip.w, fx, fy, fz, h00, h01, h02, h11, h12, h22);
    for (int r = RE; r < erows; ++r) {
        const int2 iw = __ldg(&a.st_iw[base + r * 32]);
        vbd_edge(xv, a.x[iw.x], __ldg(&a.st_rest[base + r * 32]), __int_as_float(iw.y), ip.w, fx, fy, fz, h00, h01,
                 h02, h11, h12, h22);
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) vbd_bend(xv, xb[r], wb[r], fx, fy, fz);
    for (int r = RB; r < brows; ++r) {
        const int2 iw = __ldg(&a.st_iw[bbase + r * 32]);
        vbd_bend(xv, a.x[iw.x], __int_as_float(iw.y), fx, fy, fz);
    }
#pragma unroll
    for (int o = TPV / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (!leader) return;
    if (mv.y != 0.f) {
        a.out0[v] = 0.0;
        return;
    }
    const float4 p0 = __ldcs(&a.x0[v]), vv = __ldcs(&a.vel[v]);
    const float m = p0.w, mh = m * h2inv;
    fx += -mh * ((xv.x - p0.x) - vv.x * h) + m * ip.x;
    fy += -mh * ((xv.y - p0.y) - vv.y * h) + m * ip.y;
    fz += -mh * ((xv.z - p0.z) - vv.z * h) + m * ip.z;
    a.out0[v] = (double)fx * fx + (double)fy * fy + (double)fz * fz;
}

// The probe over a resident grid: warp w takes slices w, w + nwarps, ...; lane j of a
// round looks up whether the round's j-th slice belongs to an instance being probed,
// and the warp then runs those slices only. A probe of few instances costs a couple of
// loads per warp instead of a CTA per slice.
template <int TPV, int RE, int RB>
__global__ void __launch_bounds__(128) stencil_grad32_kernel(EvalArgs a, float h, float h2inv) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    for (int round = w; round < a.nslices; round += 32 * nwarps) {
        const int s = round + lane * nwarps;
        const bool want = s < a.nslices && (!a.active || a.active[__ldg(&a.slice_inst[s])]);
        unsigned m = __ballot_sync(0xffffffffu, want);
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            grad32_slice<TPV, RE, RB>(a, round + j * nwarps, lane, h, h2inv);
        }
    }
}

// Resident CTAs of stencil_grad32_kernel, all SMs, per lanes per vertex (queried on
// first use: the eager probe at the inertial guess comes before any capture).
int grad32_ctas(int tpv) {
    static int cache[4] = {};
    const int ti = tpv == 1 ? 0 : tpv == 2 ? 1 : tpv == 4 ? 2 : 3;
    if (!cache[ti]) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        switch (tpv) {
            case 1: cache[ti] = resident_ctas(stencil_grad32_kernel<1, 6, 6>, 128, 0, sms); break;
            case 2: cache[ti] = resident_ctas(stencil_grad32_kernel<2, 3, 3>, 128, 0, sms); break;
            case 4: cache[ti] = resident_ctas(stencil_grad32_kernel<4, 2, 2>, 128, 0, sms); break;
            default: cache[ti] = resident_ctas(stencil_grad32_kernel<8, 1, 1>, 128, 0, sms); break;
        }
    }
    return cache[ti];
}

int enqueue_residual_norms(ats_cloth* c, cudaStream_t st, const int* active, bool fp32_terms) {
    EvalArgs a = eval_args(c);
    a.active = active;
    a.out0 = c->g2.p;
    if (fp32_terms) {
        const int blocks = std::min((a.nslices * 32 + 127) / 128, grad32_ctas(c->L.tpv));
        if (blocks > 0) {
            switch (c->L.tpv) {
                case 1: stencil_grad32_kernel<1, 6, 6><<<blocks, 128, 0, st>>>(a, c->h, c->h2inv); count_launch(st); break;
                case 2: stencil_grad32_kernel<2, 3, 3><<<blocks, 128, 0, st>>>(a, c->h, c->h2inv); count_launch(st); break;
                case 4: stencil_grad32_kernel<4, 2, 2><<<blocks, 128, 0, st>>>(a, c->h, c->h2inv); count_launch(st); break;
                default: stencil_grad32_kernel<8, 1, 1><<<blocks, 128, 0, st>>>(a, c->h, c->h2inv); count_launch(st); break;
            }
            ATS_CUDA(cudaGetLastError());
        }
    } else {
        ATS_CUDA(stencil_eval_launch<kEvalGrad>(c->L.tpv, a, st));
    }
    return segment_sum(c, c->g2.p, c->red_out.p, 1, st, active);
}

int enqueue_potential_pair(ats_cloth* c, const float4* y, double* gx, double* gy, cudaStream_t st) {
    const size_t nv = c->L.nv;
    if (!c->pot_vx.p) ATS_CUDA(c->pot_vx.alloc(nv));
    if (!c->pot_vy.p) ATS_CUDA(c->pot_vy.alloc(nv));
    EvalArgs a = eval_args(c);
    a.y = y;
    a.out0 = c->pot_vx.p;
    a.out1 = c->pot_vy.p;
    ATS_CUDA(stencil_eval_launch<kEvalPotPair>(c->L.tpv, a, st));
    int r;
    if ((r = segment_sum(c, c->pot_vx.p, gx, 0, st))) return r;
    return segment_sum(c, c->pot_vy.p, gy, 0, st);
}

int enqueue_potential(ats_cloth* c, double* g, cudaStream_t st) {
    if (!c->pot_vx.p) ATS_CUDA(c->pot_vx.alloc(c->L.nv));
    EvalArgs a = eval_args(c);
    a.out0 = c->pot_vx.p;
    ATS_CUDA(stencil_eval_launch<kEvalPot>(c->L.tpv, a, st));
    return segment_sum(c, c->pot_vx.p, g, 0, st);
}

// Pieces of a residual-driven frame as CUDA graphs, cached on the handle:
//   (k, 0, 0)       k = 2^j VBD iterations over the active instances;
//   (0, step, cap)  the probe of the due instances and the bookkeeping.
// A chunk of any length is the binary decomposition of its iterations, then the probe.
// Every pointer and argument baked into them is fixed for the handle (the schedule,
// tolerances and first probes are read from device memory), so a dozen graphs serve
// every frame; they are dropped with the frame graphs (ats_autotune).
int piece_graph(ats_cloth* c, int k, int step, int max_iterations, cudaGraphExec_t* out) {
    const int policy = k > 0 ? 0 : c->probe_policy;  // baked into the probe pieces
    const auto key = std::make_tuple(k, step, max_iterations, policy);
    auto it = c->chunk_graphs.find(key);
    if (it != c->chunk_graphs.end()) {
        *out = it->second;
        return ATS_OK;
    }
    cudaStream_t cs = c->capture_stream;
    cudaGraph_t g = nullptr;
    ATS_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int r = ATS_OK;
    if (k > 0) {
        r = enqueue_iterations(c, ATS_SOLVER_VBD, k, cs, c->active.p);
    } else {
        r = enqueue_residual_norms(c, cs, c->due.p, true);
        if (!r) {
            residual_check_kernel<<<1, 256, 0, cs>>>(c->red_out.p, c->norm0.p, c->active.p, c->iters.p,
                                                      c->n_active.p, c->due.p, c->L.ninst, 0, c->probe_points.p,
                                                      c->probe_idx.p, step, c->first_check.p, max_iterations,
                                                      c->tols.p, policy, c->next_due.p, c->last_it.p,
                                                      c->last_res.p); count_launch(cs);
            if (cudaGetLastError() != cudaSuccess) r = ATS_ERR_CUDA;
            if (!r) r = enqueue_compaction(c, cs);
        }
    }
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (!r) set_error(std::string("residual frame capture failed: ") + cudaGetErrorString(e));
        return r ? r : ATS_ERR_CUDA;
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    if (e == cudaSuccess) register_graph(exec, g);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        set_error(std::string("residual frame instantiate failed: ") + cudaGetErrorString(e));
        return ATS_ERR_CUDA;
    }
    c->chunk_graphs[key] = exec;
    *out = exec;
    return ATS_OK;
}

// k iterations (binary pieces), then the probe and the bookkeeping
int launch_chunk(ats_cloth* c, int k, int step, int max_iterations, cudaStream_t st) {
    int r;
    cudaGraphExec_t exec = nullptr;
    for (int bit = 1 << 20; bit > 0; bit >>= 1)
        if (k & bit) {
            if ((r = piece_graph(c, bit, 0, 0, &exec))) return r;
            ATS_CUDA(cudaGraphLaunch(exec, st));
            count_graph_launch(exec);
        }
    if ((r = piece_graph(c, 0, step, max_iterations, &exec))) return r;
    ATS_CUDA(cudaGraphLaunch(exec, st));
    count_graph_launch(exec);
    return ATS_OK;
}

int frame_to_residual_impl(ats_cloth* c, double tol, const double* tols, const int* first_check, int check_every,
                           int max_iterations, int* iterations, double* residual, cudaStream_t st,
                           const std::function<int(cudaStream_t)>& after_predict) {
    if (!c || !(tol >= 0.0) || check_every <= 0 || max_iterations < 0) {
        set_error("frame to residual: need a handle, tol >= 0, check_every > 0, max_iterations >= 0");
        return ATS_ERR_INVALID;
    }
    const int ni = c->L.ninst;
    // per-instance tolerances and first probes, on the device (the chunk graphs read them)
    if (!c->tols.p) ATS_CUDA(c->tols.alloc(ni));
    if (!c->due.p) ATS_CUDA(c->due.alloc(ni));
    if (!c->first_check.p) ATS_CUDA(c->first_check.alloc(ni));
    if (!c->next_due.p) ATS_CUDA(c->next_due.alloc(ni));
    if (!c->last_it.p) ATS_CUDA(c->last_it.alloc(ni));
    if (!c->last_res.p) ATS_CUDA(c->last_res.alloc(ni));
    if (!c->probe_idx.p) ATS_CUDA(c->probe_idx.alloc(1));
    std::vector<double> tv(ni);
    std::vector<int> fv(ni);
    for (int i = 0; i < ni; ++i) {
        tv[i] = tols ? tols[i] : tol;
        fv[i] = first_check ? std::max(1, first_check[i]) : check_every;
    }
    // probe points: every iteration count at which some instance is due (the device
    // skips instances that are not), and the cap; then the cap as a sentinel
    std::vector<char> point(max_iterations + 1, 0);
    for (int i = 0; i < ni; ++i)
        for (int k = fv[i]; k <= max_iterations; k += check_every) point[k] = 1;
    if (max_iterations > 0) point[max_iterations] = 1;
    std::vector<int> pts;
    for (int k = 1; k <= max_iterations; ++k)
        if (point[k]) pts.push_back(k);
    const int npoints = (int)pts.size();
    pts.push_back(max_iterations);
    if (c->probe_points.n < pts.size()) {
        // the chunk graphs hold the old address
        for (auto& kv : c->chunk_graphs) cudaGraphExecDestroy(kv.second);
        c->chunk_graphs.clear();
        if (c->probe_points.p) {
            cudaFree(c->probe_points.p);
            c->probe_points.p = nullptr;
            c->probe_points.n = 0;
        }
        ATS_CUDA(c->probe_points.alloc(std::max<size_t>(pts.size(), 1024)));
    }
    ATS_CUDA(cudaMemcpyAsync(c->tols.p, tv.data(), ni * sizeof(double), cudaMemcpyHostToDevice, st));
    ATS_CUDA(cudaMemcpyAsync(c->first_check.p, fv.data(), ni * sizeof(int), cudaMemcpyHostToDevice, st));
    ATS_CUDA(cudaMemcpyAsync(c->probe_points.p, pts.data(), pts.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    ATS_CUDA(cudaStreamSynchronize(st));  // the host vectors leave scope
    int r;
    for (int sub = 0; sub < c->prm.num_substep; ++sub) {
        if ((r = launch_predict(c, st))) return r;
        if ((r = enqueue_residual_norms(c, st, nullptr, true))) return r;
        if (after_predict && (r = after_predict(st))) return r;
        residual_check_kernel<<<1, 256, 0, st>>>(c->red_out.p, c->norm0.p, c->active.p, c->iters.p, c->n_active.p,
                                                  c->due.p, ni, 1, c->probe_points.p, c->probe_idx.p, check_every,
                                                  c->first_check.p, max_iterations, c->tols.p, c->probe_policy,
                                                  c->next_due.p, c->last_it.p, c->last_res.p); count_launch(st);
        ATS_CUDA(cudaGetLastError());
        if ((r = enqueue_compaction(c, st))) return r;
        list_sweep_ctas(c->L.tpv, c->block, c->list_form);  // occupancy query before any capture
        // one chunk (graphs) per probe point; the host looks at the number of active
        // instances only every kProbesPerSync points, so it rarely waits on the device
        constexpr int kProbesPerSync = 4;
        int done = 0;
        for (int p = 0; p < npoints; ++p) {
            if (p > 0 && p % kProbesPerSync == 0) {  // nothing has been probed before the first point
                ATS_CUDA(cudaMemcpyAsync(c->host_flag, c->n_active.p, sizeof(int), cudaMemcpyDeviceToHost, st));
                ATS_CUDA(cudaStreamSynchronize(st));
                if (*c->host_flag == 0) break;
            }
            if ((r = launch_chunk(c, pts[p] - done, check_every, max_iterations, st))) return r;
            done = pts[p];
        }
        if (sub + 1 == c->prm.num_substep && (iterations || residual)) {
            // report against the last substep: residual relative to ||grad G(y)|| (the
            // value of an instance's last probe)
            if (residual) {
                std::vector<double> nrm(ni), n0(ni);
                ATS_CUDA(cudaMemcpyAsync(nrm.data(), c->red_out.p, ni * sizeof(double), cudaMemcpyDeviceToHost, st));
                ATS_CUDA(cudaMemcpyAsync(n0.data(), c->norm0.p, ni * sizeof(double), cudaMemcpyDeviceToHost, st));
                ATS_CUDA(cudaStreamSynchronize(st));
                for (int i = 0; i < ni; ++i) residual[i] = n0[i] > 0.0 ? nrm[i] / n0[i] : 0.0;
            }
            if (iterations) {
                ATS_CUDA(cudaMemcpyAsync(iterations, c->iters.p, ni * sizeof(int), cudaMemcpyDeviceToHost, st));
                ATS_CUDA(cudaStreamSynchronize(st));
            }
        }
        if ((r = launch_update(c, st))) return r;
    }
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

}  // namespace ats

extern "C" {

const char* ats_last_error(void) { return g_last_error.c_str(); }

int ats_set_sweep_form(ats_cloth* c, int solver, int form) {
    if (!c || (form != 0 && form != 1) || (solver != ATS_SOLVER_VBD && solver != ATS_SOLVER_XPBD)) {
        set_error("ats_set_sweep_form: need a handle, a solver and form 0 (a launch per colour) or 1 (persistent)");
        return ATS_ERR_INVALID;
    }
    const int blocks = form == 0 ? 0
                                 : solver == ATS_SOLVER_VBD ? vbd_loop_blocks(c->L.tpv, c->block, c->device)
                                                            : c->xpbd_loop_capable;
    if (form == 1 && blocks == 0) {
        set_error("ats_set_sweep_form: the device cannot run the persistent form cooperatively");
        return ATS_ERR_INVALID;
    }
    (solver == ATS_SOLVER_VBD ? c->vbd_loop_blocks : c->xpbd_loop_blocks) = blocks;
    c->drop_graphs();  // captured frames hold the other form
    return ATS_OK;
}

int ats_set_list_sweep(ats_cloth* c, int form) {
    if (!c || form < 0 || form > 2) {
        set_error("ats_set_list_sweep: need a handle and 0 (plain), 1 (pipelined) or 2 (streamed)");
        return ATS_ERR_INVALID;
    }
    const int r = set_list_form(c, form);  // shared-memory attributes, outside any capture
    if (r) return r;
    c->drop_graphs();
    return ATS_OK;
}

int ats_set_l2_persisting(ats_cloth* c, int on) {
    if (!c || (on != 0 && on != 1)) {
        set_error("ats_set_l2_persisting: need a handle and 0 or 1");
        return ATS_ERR_INVALID;
    }
    const int r = set_l2_persisting(c, on != 0);
    if (r) return r;
    c->drop_graphs();  // captured sweeps hold the old launch attributes
    return ATS_OK;
}

int ats_selftest_bounded_waits(unsigned polls, int* barrier_status, int* mbarrier_status) {
    if (!barrier_status || !mbarrier_status || polls == 0) {
        set_error("ats_selftest_bounded_waits: need two status pointers and polls > 0");
        return ATS_ERR_INVALID;
    }
    DevBuf<unsigned> bar;
    DevBuf<int> words;
    ATS_CUDA(bar.alloc(2));
    ATS_CUDA(words.alloc(3));
    ATS_CUDA(cudaMemset(bar.p, 0, 2 * sizeof(unsigned)));
    ATS_CUDA(cudaMemset(words.p, 0, 3 * sizeof(int)));
    selftest_barrier_kernel<<<1, 32>>>(bar.p, words.p, polls);
    ATS_CUDA(cudaGetLastError());
    selftest_mbarrier_kernel<<<1, 32>>>(words.p + 1, polls);
    ATS_CUDA(cudaGetLastError());
    selftest_touch_kernel<<<1, 32>>>(words.p + 2);  // the context still runs kernels
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaDeviceSynchronize());
    int h[3] = {0, 0, 0};
    ATS_CUDA(cudaMemcpy(h, words.p, sizeof(h), cudaMemcpyDeviceToHost));
    *barrier_status = h[0] ? ATS_ERR_TIMEOUT : ATS_OK;
    *mbarrier_status = h[1] ? ATS_ERR_TIMEOUT : ATS_OK;
    if (h[2] != 12345) {
        set_error("ats_selftest_bounded_waits: a kernel after the expired waits did not run");
        return ATS_ERR_STATE;
    }
    return ATS_OK;
}

int ats_set_probe_policy(ats_cloth* c, int policy) {
    if (!c || (policy != 0 && policy != 1)) {
        set_error("ats_set_probe_policy: need a handle and policy 0 (fixed) or 1 (extrapolated)");
        return ATS_ERR_INVALID;
    }
    c->probe_policy = policy;
    return ATS_OK;
}

int ats_kernel_launches(long long* count) {
    if (!count) {
        set_error("ats_kernel_launches: null output");
        return ATS_ERR_INVALID;
    }
    *count = g_kernel_launches.load(std::memory_order_relaxed);
    return ATS_OK;
}

int ats_cloth_create(const ats_instance_desc* inst, int ninst, const ats_solver_params* prm, ats_cloth** out) {
    if (!inst || ninst <= 0 || !prm || !out) {
        set_error("ats_cloth_create: need instances, params and an output pointer");
        return ATS_ERR_INVALID;
    }
    if (!(prm->implicit_dt > 0.f) || prm->num_substep <= 0 || prm->iterations < 0) {
        set_error("ats_cloth_create: need implicit_dt > 0, num_substep > 0, iterations >= 0");
        return ATS_ERR_INVALID;
    }
    const int tpv = prm->threads_per_vertex ? prm->threads_per_vertex : 4;
    const int block = prm->block_size ? prm->block_size : 128;
    if (block % 32 || block < 32 || block > 256) {
        set_error("ats_cloth_create: block_size must be a multiple of 32 in [32, 256]");
        return ATS_ERR_INVALID;
    }
    for (int i = 0; i < ninst; ++i)
        if (!inst[i].mass || !inst[i].fixed) {
            set_error("ats_cloth_create: every instance needs mass and fixed arrays");
            return ATS_ERR_INVALID;
        }
    int r = check_device();
    if (r) return r;
    std::vector<Topology> topos(ninst);
    std::vector<ats_instance_desc> descs(inst, inst + ninst);
    std::string err;
    {
        // instances are independent: build their topologies on a few host threads
        std::vector<std::string> errs(ninst);
        std::vector<char> ok(ninst, 1);
        const int nthreads = std::max(1, std::min(ninst, (int)std::thread::hardware_concurrency()));
        std::atomic<int> next{0};
        auto work = [&] {
            for (int i = next++; i < ninst; i = next++) ok[i] = build_topology(inst[i], topos[i], errs[i]);
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nthreads; ++t) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        for (int i = 0; i < ninst; ++i)
            if (!ok[i]) {
                set_error("ats_cloth_create: instance " + std::to_string(i) + ": " + errs[i]);
                return ATS_ERR_INVALID;
            }
    }
    std::unique_ptr<ats_cloth> c(new (std::nothrow) ats_cloth());
    if (!c) {
        set_error("ats_cloth_create: out of memory");
        return ATS_ERR_NOMEM;
    }
    if (!build_layout(topos, descs, prm->gravity, tpv, c->L, err)) {
        set_error("ats_cloth_create: " + err);
        return ATS_ERR_INVALID;
    }
    topos.clear();
    c->prm = *prm;
    c->prm.threads_per_vertex = tpv;
    c->prm.block_size = block;
    c->block = block;
    c->h = prm->implicit_dt / float(prm->num_substep);
    c->h2inv = 1.f / (c->h * c->h);
    c->damp = std::exp(-prm->damping * c->h);
    ATS_CUDA(cudaGetDevice(&c->device));
    const Layout& L = c->L;
    const size_t nv = L.nv;
    if ((r = upload(c->x, L.x0, nv)) || (r = upload(c->x0, L.x0, nv)) || (r = upload(c->vel, L.vel, nv)) ||
        (r = upload(c->vm, L.vm, nv)) || (r = upload(c->inst, L.inst, L.ninst)))
        return r;
    if ((r = upload_stencil(c.get()))) return r;
    if ((r = upload(c->xs_edge, L.xs_edge, L.xs_rest.size())) || (r = upload(c->xs_rest, L.xs_rest, L.xs_rest.size())) ||
        (r = upload(c->xs_k, L.xs_k, L.xs_k.size())))
        return r;
    ATS_CUDA(c->xs_lambda.alloc(L.xs_rest.size()));
    if ((r = upload(c->xb_idx, L.xb_idx, L.xb_idx.size() / 4)) || (r = upload(c->xb_q, L.xb_q, L.xb_q.size() / 4)))
        return r;
    ATS_CUDA(c->xb_lambda.alloc(L.xb_idx.size() / 4));
    // the persistent XPBD kernel: colour offsets on the device, barrier state, and one
    // 1024-thread block per SM when the device runs cooperative launches of it
    if ((r = upload(c->xs_color_d, L.xs_color, L.xs_color.size())) ||
        (r = upload(c->xb_color_d, L.xb_color, L.xb_color.size())))
        return r;
    ATS_CUDA(c->loop_bar.alloc(2));
    ATS_CUDA(c->loop_err.alloc(1));
    ATS_CUDA(cudaMemset(c->loop_bar.p, 0, 2 * sizeof(unsigned)));
    ATS_CUDA(cudaMemset(c->loop_err.p, 0, sizeof(int)));
    {
        int coop = 0, sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, xpbd_loop_kernel, kXpbdLoopThreads, 0) != cudaSuccess)
            per_sm = 0;
        c->xpbd_loop_capable = coop && per_sm >= 1 ? sms : 0;
        c->xpbd_loop_blocks = 0;  // per-colour launches until ats_autotune or ats_set_sweep_form chooses
    }
    if ((r = upload(c->en_edge, L.en_edge, L.en_rest.size())) || (r = upload(c->en_rest, L.en_rest, L.en_rest.size())) ||
        (r = upload(c->en_k, L.en_k, L.en_k.size())) || (r = upload(c->en_bend, L.en_bend, L.en_kb.size())) ||
        (r = upload(c->en_q, L.en_q, L.en_q.size())) || (r = upload(c->en_kb, L.en_kb, L.en_kb.size())))
        return r;
    if ((r = upload(c->inst_seg, L.inst_vbegin, L.inst_vbegin.size()))) return r;
    if ((r = upload(c->to_caller, L.to_caller, nv))) return r;
    if ((r = upload(c->feat_nb, L.feat_nb, L.feat_nb.size())) || (r = upload(c->feat_len, L.feat_len, L.feat_len.size())) ||
        (r = upload(c->inst_eseg, L.inst_eseg, L.inst_eseg.size())) ||
        (r = upload(c->inst_bseg, L.inst_bseg, L.inst_bseg.size())))
        return r;
    ATS_CUDA(c->io_x.alloc(3 * nv));
    ATS_CUDA(c->io_v.alloc(3 * nv));
    ATS_CUDA(c->partial.alloc(3 * (size_t)kRedBlocks));
    ATS_CUDA(c->seg_partial.alloc((size_t)kSegChunks * L.ninst));
    ATS_CUDA(c->red_out.alloc(std::max(3, L.ninst)));
    ATS_CUDA(c->g2.alloc(nv));
    ATS_CUDA(c->norm0.alloc(L.ninst));
    ATS_CUDA(c->active.alloc(L.ninst));
    ATS_CUDA(c->iters.alloc(L.ninst));
    ATS_CUDA(c->n_active.alloc(1));
    ATS_CUDA(cudaHostAlloc((void**)&c->host_flag, sizeof(int), cudaHostAllocDefault));
    ATS_CUDA(cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking));
    ATS_CUDA(cudaDeviceSynchronize());
    *out = c.release();
    return ATS_OK;
}

int ats_cloth_destroy(ats_cloth* c) {
    if (!c) return ATS_OK;
    cudaDeviceSynchronize();
    l2_keep_release(c);
    delete c;
    return ATS_OK;
}

int ats_cloth_query(const ats_cloth* c, ats_cloth_info* info) {
    if (!c || !info) {
        set_error("ats_cloth_query: null argument");
        return ATS_ERR_INVALID;
    }
    info->num_instances = c->L.ninst;
    info->num_verts = c->L.nv;
    info->num_edges = c->L.ne;
    info->num_bending_edges = c->L.nb;
    info->num_vertex_colors = c->L.n_vcolors;
    info->num_stretch_colors = c->L.n_scolors;
    info->num_bending_colors = c->L.n_bcolors;
    info->threads_per_vertex = c->L.tpv;
    info->block_size = c->block;
    info->stencil_slots = (int)c->L.st_rest.size();
    info->device_bytes = (long long)c->device_bytes();
    info->vbd_form = c->vbd_loop_blocks > 0 ? 1 : 0;
    info->xpbd_form = c->xpbd_loop_blocks > 0 ? 1 : 0;
    info->list_form = c->list_form;
    info->tune_source = c->tune_source;
    info->l2_persisting = c->l2_keep ? 1 : 0;
    long long sb = 64LL * c->L.nv;
    for (size_t k = 0; k + 3 < c->L.slices.size(); k += 4) {
        const int rows = c->L.slices[k + 3] & 0xffff, erows = c->L.slices[k + 3] >> 16;
        sb += 32LL * (8 * rows + 4 * erows) + 28;
    }
    info->sweep_layout_bytes = sb;
    return ATS_OK;
}

int ats_cloth_vertex_order(const ats_cloth* c, int* layout_of_caller) {
    if (!c || !layout_of_caller) {
        set_error("ats_cloth_vertex_order: null argument");
        return ATS_ERR_INVALID;
    }
    std::memcpy(layout_of_caller, c->L.to_layout.data(), c->L.nv * sizeof(int));
    return ATS_OK;
}

int ats_set_state(ats_cloth* c, const float* x, const float* v, ats_stream stream) {
    if (!c || !x) {
        set_error("ats_set_state: need a handle and positions");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    const int n = c->L.nv;
    ATS_CUDA(cudaMemcpyAsync(c->io_x.p, x, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    if (v) ATS_CUDA(cudaMemcpyAsync(c->io_v.p, v, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    scatter_state_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->io_x.p, c->io_v.p, c->to_caller.p, c->x.p, c->x0.p,
                                                          c->vel.p, n, v ? 1 : 0); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_set_positions(ats_cloth* c, const float* x, ats_stream stream) {
    if (!c || !x) {
        set_error("ats_set_positions: need a handle and positions");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    const int n = c->L.nv;
    ATS_CUDA(cudaMemcpyAsync(c->io_x.p, x, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    scatter_positions_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->io_x.p, c->to_caller.p, c->x.p, n); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

// A grid barrier of the persistent XPBD kernel that ran out of polls leaves loop_err
// set (the kernel returned early); the next state read reports it once and clears it.
static int check_loop_error(ats_cloth* c, cudaStream_t st) {
    if (!c->loop_err.p) return ATS_OK;
    ATS_CUDA(cudaMemcpyAsync(c->host_flag, c->loop_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    if (*c->host_flag == 0) return ATS_OK;
    ATS_CUDA(cudaMemsetAsync(c->loop_err.p, 0, sizeof(int), st));
    ATS_CUDA(cudaStreamSynchronize(st));
    set_error("XPBD persistent kernel: a grid barrier wait expired; the frame stopped early");
    return ATS_ERR_TIMEOUT;
}

static int read_back(ats_cloth* c, const float4* src, float* dst, float* staging, cudaStream_t st) {
    const int n = c->L.nv;
    gather_state_kernel<<<(n + 255) / 256, 256, 0, st>>>(src, c->to_caller.p, staging, n); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaMemcpyAsync(dst, staging, 12 * (size_t)n, cudaMemcpyDeviceToHost, st));
    return ATS_OK;
}

int ats_async_fork(ats_cloth* c, ats_stream stream) {
    if (!c) {
        set_error("ats_async_fork: null handle");
        return ATS_ERR_INVALID;
    }
    if (!c->async_begin.p) ATS_CUDA(c->async_begin.alloc(c->L.nv));
    ATS_CUDA(cudaMemcpyAsync(c->async_begin.p, c->x.p, c->x.bytes(), cudaMemcpyDeviceToDevice, S(stream)));
    return ATS_OK;
}

int ats_async_merge(ats_cloth* c, const float* other, float weight, ats_stream stream) {
    if (!c || !other) {
        set_error("ats_async_merge: null argument");
        return ATS_ERR_INVALID;
    }
    if (!c->async_begin.p) {
        set_error("ats_async_merge: no fork point (call ats_async_fork first)");
        return ATS_ERR_INVALID;
    }
    const int n = c->L.nv;
    cudaStream_t st = S(stream);
    ATS_CUDA(cudaMemcpyAsync(c->io_x.p, other, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    async_merge_kernel<<<(n + 255) / 256, 256, 0, st>>>(c->x.p, c->async_begin.p, c->io_x.p, c->to_caller.p, n, weight); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_get_state(ats_cloth* c, float* x, float* v, ats_stream stream) {
    if (!c || !x) {
        set_error("ats_get_state: need a handle and an output array");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = read_back(c, c->x0.p, x, c->io_x.p, st);
    if (!r && v) r = read_back(c, c->vel.p, v, c->io_v.p, st);
    if (r) return r;
    ATS_CUDA(cudaStreamSynchronize(st));
    return check_loop_error(c, st);
}

int ats_get_positions(ats_cloth* c, float* x, ats_stream stream) {
    if (!c || !x) {
        set_error("ats_get_positions: need a handle and an output array");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = read_back(c, c->x.p, x, c->io_x.p, st);
    if (r) return r;
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_set_accel(ats_cloth* c, const float* accel, ats_stream stream) {
    if (!c || !accel) {
        set_error("ats_set_accel: null argument");
        return ATS_ERR_INVALID;
    }
    for (int i = 0; i < c->L.ninst; ++i)
        for (int k = 0; k < 3; ++k) c->L.inst[4 * i + k] = accel[3 * i + k];
    ATS_CUDA(cudaMemcpyAsync(c->inst.p, c->L.inst.data(), c->L.inst.size() * sizeof(float), cudaMemcpyHostToDevice,
                             S(stream)));
    ATS_CUDA(cudaStreamSynchronize(S(stream)));
    return ATS_OK;
}

int ats_predict_position(ats_cloth* c, ats_stream stream) {
    if (!c) { set_error("ats_predict_position: null handle"); return ATS_ERR_INVALID; }
    return launch_predict(c, S(stream));
}

int ats_vbd_color_sweep(ats_cloth* c, int color, ats_stream stream) {
    if (!c || color < 0 || color >= c->L.n_vcolors) {
        set_error("ats_vbd_color_sweep: null handle or colour out of range");
        return ATS_ERR_INVALID;
    }
    return launch_sweep(c, color, S(stream));
}

int ats_vbd_iterations(ats_cloth* c, int iterations, ats_stream stream) {
    if (!c || iterations < 0) {
        set_error("ats_vbd_iterations: null handle or negative count");
        return ATS_ERR_INVALID;
    }
    return enqueue_iterations(c, ATS_SOLVER_VBD, iterations, S(stream));
}

int ats_update_velocity(ats_cloth* c, ats_stream stream) {
    if (!c) { set_error("ats_update_velocity: null handle"); return ATS_ERR_INVALID; }
    return launch_update(c, S(stream));
}

int ats_xpbd_reset_constraints(ats_cloth* c, ats_stream stream) {
    if (!c) { set_error("ats_xpbd_reset_constraints: null handle"); return ATS_ERR_INVALID; }
    return launch_reset(c, S(stream));
}

int ats_xpbd_stretch_color(ats_cloth* c, int color, ats_stream stream) {
    if (!c || color < 0 || color >= c->L.n_scolors) {
        set_error("ats_xpbd_stretch_color: null handle or colour out of range");
        return ATS_ERR_INVALID;
    }
    return launch_xpbd_stretch(c, color, S(stream));
}

int ats_xpbd_bending_color(ats_cloth* c, int color, ats_stream stream) {
    if (!c || color < 0 || color >= c->L.n_bcolors) {
        set_error("ats_xpbd_bending_color: null handle or colour out of range");
        return ATS_ERR_INVALID;
    }
    return launch_xpbd_bending(c, color, S(stream));
}

int ats_frame(ats_cloth* c, int solver, ats_stream stream) {
    if (!c || (solver != ATS_SOLVER_VBD && solver != ATS_SOLVER_XPBD)) {
        set_error("ats_frame: null handle or unknown solver");
        return ATS_ERR_INVALID;
    }
    return enqueue_frame(c, solver, S(stream));
}

int ats_frame_graph(ats_cloth* c, int solver, ats_stream stream) {
    if (!c || (solver != ATS_SOLVER_VBD && solver != ATS_SOLVER_XPBD)) {
        set_error("ats_frame_graph: null handle or unknown solver");
        return ATS_ERR_INVALID;
    }
    if (!c->graph[solver]) {
        cudaGraph_t g = nullptr;
        ATS_CUDA(cudaStreamBeginCapture(c->capture_stream, cudaStreamCaptureModeThreadLocal));
        int r = enqueue_frame(c, solver, c->capture_stream);
        cudaError_t e = cudaStreamEndCapture(c->capture_stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) {
            set_error(std::string("ats_frame_graph: capture failed: ") + cudaGetErrorString(e));
            return ATS_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&c->graph[solver], g, 0);
        if (e == cudaSuccess) register_graph(c->graph[solver], g);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            set_error(std::string("ats_frame_graph: instantiate failed: ") + cudaGetErrorString(e));
            return ATS_ERR_CUDA;
        }
    }
    ATS_CUDA(cudaGraphLaunch(c->graph[solver], S(stream)));
    count_graph_launch(c->graph[solver]);
    return ATS_OK;
}

}  // extern "C"

namespace ats {
// The autotuner's choices per (GPU, mesh class), shared by the handles of a process and
// saved to / loaded from a text file by ats_autotune_cache_save / _load. The mesh class
// is what the choices depend on: the vertex and instance counts (power-of-two buckets)
// and the colour counts of both solvers.
struct TuneChoice {
    int tpv, block, vbd_form, list_form, xpbd_form, l2;
};
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tune_cache;

int floor_log2(long long v) {
    int k = 0;
    while (v > 1) {
        v >>= 1;
        ++k;
    }
    return k;
}

std::string tune_key(const ats_cloth* c) {
    cudaDeviceProp p;
    std::string dev = "unknown";
    int sms = 0;
    if (cudaGetDeviceProperties(&p, c->device) == cudaSuccess) {
        dev = p.name;
        sms = p.multiProcessorCount;
    }
    for (char& ch : dev)
        if (ch == ' ' || ch == '|' || ch == '\n') ch = '_';
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s|%d|v%d|i%d|c%d|s%d|b%d", dev.c_str(), sms, floor_log2(c->L.nv),
                  floor_log2(c->L.ninst), c->L.n_vcolors, c->L.n_scolors, c->L.n_bcolors);
    return buf;
}

// Applies cached choices to a handle: its layout for the lanes per vertex, the block
// size and the forms (a persistent form only where the device can run it).
int apply_tuning(ats_cloth* c, const TuneChoice& t) {
    std::string err;
    if (t.tpv != c->L.tpv) {
        int r;
        if (!build_slices(c->L, t.tpv, err)) {
            set_error("ats_autotune: " + err);
            return ATS_ERR_INVALID;
        }
        if ((r = upload_stencil(c))) return r;
    }
    c->block = t.block;
    c->vbd_loop_blocks = t.vbd_form ? vbd_loop_blocks(c->L.tpv, c->block, c->device) : 0;
    set_list_form(c, t.list_form);
    if (set_l2_persisting(c, t.l2 != 0)) set_l2_persisting(c, false);  // no persisting L2 on this device
    c->xpbd_loop_blocks = t.xpbd_form ? c->xpbd_loop_capable : 0;
    c->prm.threads_per_vertex = c->L.tpv;
    c->prm.block_size = c->block;
    c->drop_graphs();
    return ATS_OK;
}
}  // namespace ats

extern "C" {

int ats_autotune_cache_size(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return (int)g_tune_cache.size();
}

void ats_autotune_cache_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.clear();
}

int ats_autotune_cache_save(const char* path) {
    if (!path) {
        set_error("ats_autotune_cache_save: null path");
        return ATS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    FILE* f = std::fopen(path, "w");
    if (!f) {
        set_error(std::string("ats_autotune_cache_save: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    std::fprintf(f, "ats-autotune 2\n");
    for (const auto& kv : g_tune_cache)
        std::fprintf(f, "%s %d %d %d %d %d %d\n", kv.first.c_str(), kv.second.tpv, kv.second.block, kv.second.vbd_form,
                     kv.second.list_form, kv.second.xpbd_form, kv.second.l2);
    const bool ok = std::fclose(f) == 0;
    if (!ok) {
        set_error(std::string("ats_autotune_cache_save: write failed: ") + path);
        return ATS_ERR_INVALID;
    }
    return ATS_OK;
}

int ats_autotune_cache_load(const char* path) {
    if (!path) {
        set_error("ats_autotune_cache_load: null path");
        return ATS_ERR_INVALID;
    }
    FILE* f = std::fopen(path, "r");
    if (!f) {
        set_error(std::string("ats_autotune_cache_load: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    char line[512];
    std::map<std::string, TuneChoice> got;
    bool header = false, bad = false;
    while (std::fgets(line, sizeof(line), f)) {
        if (!header) {
            header = std::strncmp(line, "ats-autotune 2", 14) == 0;
            if (!header) bad = true;
            if (bad) break;
            continue;
        }
        char key[400];
        TuneChoice t;
        if (std::sscanf(line, "%399s %d %d %d %d %d %d", key, &t.tpv, &t.block, &t.vbd_form, &t.list_form, &t.xpbd_form,
                        &t.l2) != 7 ||
            !(t.tpv == 1 || t.tpv == 2 || t.tpv == 4 || t.tpv == 8) || !(t.block == 64 || t.block == 128 || t.block == 256) ||
            t.vbd_form < 0 || t.vbd_form > 1 || t.list_form < 0 || t.list_form > 2 || t.xpbd_form < 0 || t.xpbd_form > 1 ||
            t.l2 < 0 || t.l2 > 1) {
            bad = true;
            break;
        }
        got[key] = t;
    }
    std::fclose(f);
    if (bad || !header) {
        set_error(std::string("ats_autotune_cache_load: malformed file ") + path);
        return ATS_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& kv : got) g_tune_cache[kv.first] = kv.second;
    return ATS_OK;
}

int ats_autotune(ats_cloth* c, int iterations, ats_stream stream, int* out_tpv, int* out_block) {
    if (!c || iterations <= 0) {
        set_error("ats_autotune: null handle or iterations <= 0");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    // a choice made before for this GPU and mesh class: applied without timing
    const std::string key = tune_key(c);
    {
        TuneChoice t{};
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune_cache.find(key);
            if (it != g_tune_cache.end()) {
                t = it->second;
                hit = true;
            }
        }
        if (hit) {
            const int r = apply_tuning(c, t);
            if (r) return r;
            c->tune_source = 2;
            if (out_tpv) *out_tpv = c->L.tpv;
            if (out_block) *out_block = c->block;
            return ATS_OK;
        }
    }
    // keep the iterate: the trial sweeps move it
    DevBuf<float4> saved;
    ATS_CUDA(saved.alloc(c->L.nv));
    ATS_CUDA(cudaMemcpyAsync(saved.p, c->x.p, c->x.bytes(), cudaMemcpyDeviceToDevice, st));
    cudaEvent_t e0, e1;
    ATS_CUDA(cudaEventCreate(&e0));
    ATS_CUDA(cudaEventCreate(&e1));
    const int tpvs[4] = {1, 2, 4, 8};
    const int blocks[3] = {64, 128, 256};
    float best = 1e30f;
    int best_tpv = c->L.tpv, best_block = c->block;
    std::string err;
    int r = ATS_OK;
    c->vbd_loop_blocks = 0;  // the one-wave launches first
    // the fastest of three timings of `iterations` iterations (short runs are noisy)
    auto time_iterations = [&](float& ms) -> int {
        int rr;
        if ((rr = enqueue_iterations(c, ATS_SOLVER_VBD, 1, st))) return rr;  // warm-up
        ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, st);
            if ((rr = enqueue_iterations(c, ATS_SOLVER_VBD, iterations, st))) return rr;
            cudaEventRecord(e1, st);
            cudaError_t ce = cudaEventSynchronize(e1);
            if (ce != cudaSuccess) {
                set_error(std::string("ats_autotune: ") + cudaGetErrorString(ce));
                return ATS_ERR_CUDA;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        return ATS_OK;
    };
    for (int tpv : tpvs) {
        if (!build_slices(c->L, tpv, err) || (r = upload_stencil(c))) {
            if (!r) {
                set_error("ats_autotune: " + err);
                r = ATS_ERR_INVALID;
            }
            break;
        }
        for (int b : blocks) {
            c->block = b;
            float ms = 1e30f;
            if ((r = time_iterations(ms))) break;
            if (ms < best) {
                best = ms;
                best_tpv = tpv;
                best_block = b;
            }
        }
        if (r) break;
    }
    if (!r && (!build_slices(c->L, best_tpv, err) || (r = upload_stencil(c)))) {
        if (!r) {
            set_error("ats_autotune: " + err);
            r = ATS_ERR_INVALID;
        }
    }
    c->block = best_block;
    // then the persistent form at the chosen shape: kept where it is faster
    if (!r) {
        const int loop_blocks = vbd_loop_blocks(c->L.tpv, c->block, c->device);
        if (loop_blocks > 0) {
            c->vbd_loop_blocks = loop_blocks;
            float ms = 1e30f;
            r = time_iterations(ms);
            if (r || ms >= best) c->vbd_loop_blocks = 0;
        }
    }
    // the list sweep of the residual-driven frames, its four forms, over every
    // instance's slices (all instances active): the fastest of three timings each
    if (!r && c->L.ninst > 0) {
        std::vector<int> ones(c->L.ninst, 1);
        ATS_CUDA(cudaMemcpyAsync(c->active.p, ones.data(), ones.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        if (!(r = enqueue_compaction(c, st))) {
            // forms 0-2, then the fastest with the positions persisting in L2 (slot 3 here)
            float t_form[4] = {1e30f, 1e30f, 1e30f, 1e30f};
            int best_form = 0;
            set_l2_persisting(c, false);
            for (int form = 0; form < 4 && !r; ++form) {
                if (form == 3) {
                    for (int f = 1; f < 3; ++f)
                        if (t_form[f] < t_form[best_form]) best_form = f;
                    if (set_l2_persisting(c, true)) break;  // no persisting L2 on this device
                }
                set_list_form(c, form < 3 ? form : best_form);
                if ((r = enqueue_iterations(c, ATS_SOLVER_VBD, 1, st, c->active.p))) break;
                for (int rep = 0; rep < 3; ++rep) {
                    cudaEventRecord(e0, st);
                    if ((r = enqueue_iterations(c, ATS_SOLVER_VBD, iterations, st, c->active.p))) break;
                    cudaEventRecord(e1, st);
                    if (cudaEventSynchronize(e1) != cudaSuccess) {
                        set_error("ats_autotune: list sweep timing failed");
                        r = ATS_ERR_CUDA;
                        break;
                    }
                    float t = 0.f;
                    cudaEventElapsedTime(&t, e0, e1);
                    t_form[form] = std::min(t_form[form], t);
                }
            }
            if (!r) {
                for (int f = 1; f < 3; ++f)
                    if (t_form[f] < t_form[best_form]) best_form = f;
                set_list_form(c, best_form);
                set_l2_persisting(c, t_form[3] < t_form[best_form]);
            }
        }
        ATS_CUDA(cudaStreamSynchronize(st));  // the host vector leaves scope
    }
    // XPBD iterations: per-colour launches against the persistent kernel (the fastest of
    // three timings each); lambda is reset afterwards by every frame, x restored below
    if (!r && c->xpbd_loop_capable > 0 && c->L.n_scolors + c->L.n_bcolors > 0) {
        float t_form[2] = {1e30f, 1e30f};
        for (int form = 0; form < 2 && !r; ++form) {
            c->xpbd_loop_blocks = form ? c->xpbd_loop_capable : 0;
            if ((r = enqueue_iterations(c, ATS_SOLVER_XPBD, 1, st))) break;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, st);
                if ((r = enqueue_iterations(c, ATS_SOLVER_XPBD, iterations, st))) break;
                cudaEventRecord(e1, st);
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    set_error("ats_autotune: XPBD timing failed");
                    r = ATS_ERR_CUDA;
                    break;
                }
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                t_form[form] = std::min(t_form[form], t);
            }
        }
        c->xpbd_loop_blocks = !r && t_form[1] < t_form[0] ? c->xpbd_loop_capable : 0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->prm.threads_per_vertex = c->L.tpv;
    c->prm.block_size = best_block;
    c->drop_graphs();
    ATS_CUDA(cudaMemcpyAsync(c->x.p, saved.p, c->x.bytes(), cudaMemcpyDeviceToDevice, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    if (r) return r;
    c->tune_source = 1;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = TuneChoice{c->L.tpv, c->block, c->vbd_loop_blocks > 0 ? 1 : 0, c->list_form,
                                       c->xpbd_loop_blocks > 0 ? 1 : 0, c->l2_keep ? 1 : 0};
    }
    if (out_tpv) *out_tpv = c->L.tpv;
    if (out_block) *out_block = c->block;
    return ATS_OK;
}

int ats_potential(ats_cloth* c, double* out, ats_stream stream) {
    if (!c || !out) {
        set_error("ats_potential: null argument");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = enqueue_potential(c, c->red_out.p, st);
    if (r) return r;
    ATS_CUDA(cudaMemcpyAsync(out, c->red_out.p, c->L.ninst * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_energy(ats_cloth* c, double* out3, ats_stream stream) {
    if (!c || !out3) {
        set_error("ats_energy: null argument");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    EnergyArgs a;
    a.x = c->x.p;
    a.x0 = c->x0.p;
    a.vel = c->vel.p;
    a.vm = c->vm.p;
    a.inst = c->inst.p;
    a.nv = c->L.nv;
    a.edge = c->en_edge.p;
    a.rest = c->en_rest.p;
    a.kst = c->en_k.p;
    a.ne = c->L.ne;
    a.bend = c->en_bend.p;
    a.q16 = c->en_q.p;
    a.kb = c->en_kb.p;
    a.nb = c->L.nb;
    a.h = (double)c->h;
    a.partial = c->partial.p;
    energy_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    sum_partials3_kernel<<<1, kRedThreads, 0, st>>>(c->partial.p, kRedBlocks, c->red_out.p); count_launch(st);
    ATS_CUDA(cudaGetLastError());
    ATS_CUDA(cudaMemcpyAsync(out3, c->red_out.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

int ats_frame_to_residual(ats_cloth* c, double tol, int check_every, int max_iterations, int* iterations,
                          double* residual, ats_stream stream) {
    if (!c) {
        set_error("ats_frame_to_residual: null handle");
        return ATS_ERR_INVALID;
    }
    return frame_to_residual_impl(c, tol, nullptr, nullptr, check_every, max_iterations, iterations, residual,
                                  S(stream), nullptr);
}

int ats_frame_to_residuals(ats_cloth* c, const double* tols, const int* first_check, int check_every,
                           int max_iterations, int* iterations, double* residual, ats_stream stream) {
    if (!c || !tols) {
        set_error("ats_frame_to_residuals: need a handle and one tolerance per instance");
        return ATS_ERR_INVALID;
    }
    return frame_to_residual_impl(c, 0.0, tols, first_check, check_every, max_iterations, iterations, residual,
                                  S(stream), nullptr);
}

int ats_residual(ats_cloth* c, double* out, ats_stream stream) {
    if (!c || !out) {
        set_error("ats_residual: null argument");
        return ATS_ERR_INVALID;
    }
    cudaStream_t st = S(stream);
    int r = enqueue_residual_norms(c, st);
    if (r) return r;
    ATS_CUDA(cudaMemcpyAsync(out, c->red_out.p, c->L.ninst * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATS_CUDA(cudaStreamSynchronize(st));
    return ATS_OK;
}

}  // extern "C"
