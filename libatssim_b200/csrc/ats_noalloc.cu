// ats_noalloc.cu -- FP64 cloth energy that allocates no device memory.
//
// Who needs this: programs whose GPU memory is handed out by their own allocator
// (a game engine or simulation framework that reserves the device heap at start-up
// and forbids other allocations), and per-frame loops that cannot afford
// cudaMalloc / cudaFree, which may synchronise the whole device. Such callers own
// the input and output buffers already; ats_energy_noalloc reads those and keeps
// its block partial sums in a fixed static device array of this file instead of a
// handle's cudaMalloc'ed scratch.
//
// Limits and sharing:
//   * at most kNoallocMaxElements vertices, edges and bending edges per call
//     (kNoallocMaxPartials blocks x kNoallocChunk elements); larger calls are
//     rejected with ATS_ERR_INVALID before anything is launched;
//   * the array (3 x kNoallocMaxPartials doubles = 96 KiB) lives on every GPU that
//     loads the library until the process exits;
//   * every call on a device uses the same array and leaves its partial sums in it.
//     Each call writes every partial it later reads, so nothing needs clearing, but
//     two calls whose kernels overlap on the GPU (different streams, or different
//     host threads) race on the array and may return wrong sums.

#include <cuda_runtime.h>

#include <string>

#include "../../include/ats_cloth.h"

namespace ats {
void set_error(const std::string& msg);
}

namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocChunk = 2048;         // elements of one term per block
constexpr int kNoallocMaxPartials = 4096;   // blocks per term
constexpr long long kNoallocMaxElements = (long long)kNoallocChunk * kNoallocMaxPartials;  // 8,388,608

// Partial sums: [term][block], term 0 inertia, 1 stretch, 2 bending.
static __device__ __align__(256) double g_noalloc_partials[3 * kNoallocMaxPartials];

// Device address of g_noalloc_partials on the current device. The host-side symbol
// is only a stand-in, never a device address, so every call asks the runtime for the
// address: once the module is loaded the lookup is cheap, and a cached pointer would
// go stale after cudaDeviceReset or a rebuilt primary context reloads the module.
int partials_address(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
        ats::set_error(std::string("ats_energy_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return ATS_ERR_CUDA;
    }
    *out = (double*)p;
    return ATS_OK;
}

__device__ __forceinline__ double block_sum_noalloc(double v, double* sh) {
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

struct NoallocArgs {
    const float* x;
    const float* x_start;
    const float* v;
    const float* mass;
    const unsigned char* fixed;
    int nv;
    const int* edges;
    const float* rest;
    int ne;
    const int* bending;
    const float* q;
    int nb;
    float k_stretch, k_bend;
    double ax, ay, az, h;
    double* partials;  // device address of g_noalloc_partials
};

// Block b sums elements [b*kNoallocChunk, (b+1)*kNoallocChunk) of each term, the
// same per-term formulas as the handle's energy kernel
// (Energy::compute_energy_*, xpbd_constraints.h:2079-2214, all in FP64).
__global__ void __launch_bounds__(kNoallocThreads) energy_noalloc_kernel(NoallocArgs a) {
    __shared__ double sh[kNoallocThreads];
    const int b = blockIdx.x;
    const int lo = b * kNoallocChunk;
    double ei = 0.0, es = 0.0, eb = 0.0;
    const int hi_v = min(a.nv, lo + kNoallocChunk);
    for (int i = lo + threadIdx.x; i < hi_v; i += kNoallocThreads) {
        const bool pinned = a.fixed[i] != 0;
        const double ax = pinned ? 0.0 : a.ax, ay = pinned ? 0.0 : a.ay, az = pinned ? 0.0 : a.az;
        const float* p = a.x + 3 * (size_t)i;
        const float* q0 = a.x_start + 3 * (size_t)i;
        const float* vv = a.v + 3 * (size_t)i;
        const double dx = (double)p[0] - ((double)q0[0] + a.h * vv[0] + a.h * a.h * ax);
        const double dy = (double)p[1] - ((double)q0[1] + a.h * vv[1] + a.h * a.h * ay);
        const double dz = (double)p[2] - ((double)q0[2] + a.h * vv[2] + a.h * a.h * az);
        ei += (double)a.mass[i] / (2.0 * a.h * a.h) * (dx * dx + dy * dy + dz * dz);
    }
    const int hi_e = min(a.ne, lo + kNoallocChunk);
    for (int i = lo + threadIdx.x; i < hi_e; i += kNoallocThreads) {
        const float* p0 = a.x + 3 * (size_t)a.edges[2 * i];
        const float* p1 = a.x + 3 * (size_t)a.edges[2 * i + 1];
        const double dx = (double)p1[0] - p0[0], dy = (double)p1[1] - p0[1], dz = (double)p1[2] - p0[2];
        const double l2 = dx * dx + dy * dy + dz * dz;
        if (l2 < 1e-8) continue;
        const double C = sqrt(l2) - (double)a.rest[i];
        es += 0.5 * (double)a.k_stretch * C * C;
    }
    const int hi_b = min(a.nb, lo + kNoallocChunk);
    for (int i = lo + threadIdx.x; i < hi_b; i += kNoallocThreads) {
        double p[4][3];
        for (int j = 0; j < 4; ++j) {
            const float* t = a.x + 3 * (size_t)a.bending[4 * i + j];
            p[j][0] = t[0];
            p[j][1] = t[1];
            p[j][2] = t[2];
        }
        const float* Q = a.q + 16 * (size_t)i;
        double s = 0.0;
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r)
                s += (double)Q[4 * c + r] * (p[c][0] * p[r][0] + p[c][1] * p[r][1] + p[c][2] * p[r][2]);
        eb += 0.5 * (double)a.k_bend * s;
    }
    const double si = block_sum_noalloc(ei, sh);
    const double ss = block_sum_noalloc(es, sh);
    const double sb = block_sum_noalloc(eb, sh);
    if (threadIdx.x == 0) {
        a.partials[0 * kNoallocMaxPartials + b] = si;
        a.partials[1 * kNoallocMaxPartials + b] = ss;
        a.partials[2 * kNoallocMaxPartials + b] = sb;
    }
}

// Adds the partials of each term in block order; out3 is the caller's device array.
__global__ void __launch_bounds__(kNoallocThreads) energy_noalloc_final_kernel(const double* partials, int nblk_v,
                                                                              int nblk_e, int nblk_b, double* out3) {
    __shared__ double sh[kNoallocThreads];
    const int n[3] = {nblk_v, nblk_e, nblk_b};
    for (int t = 0; t < 3; ++t) {
        double v = 0.0;
        for (int i = threadIdx.x; i < n[t]; i += kNoallocThreads) v += partials[t * kNoallocMaxPartials + i];
        const double s = block_sum_noalloc(v, sh);
        if (threadIdx.x == 0) out3[t] = s;
    }
}

}  // namespace

extern "C" int ats_energy_noalloc(const float* x, const float* x_start, const float* v, const float* mass,
                                  const unsigned char* fixed, int num_verts, const int* edges, const float* rest_length,
                                  int num_edges, const int* bending, const float* q, int num_bending_edges,
                                  float k_stretch, float k_bend, const float* accel, float h, double* out3,
                                  ats_stream stream) {
    if (!x || !x_start || !v || !mass || !fixed || !accel || !out3 || num_verts <= 0 || num_edges < 0 ||
        num_bending_edges < 0 || (num_edges > 0 && (!edges || !rest_length)) ||
        (num_bending_edges > 0 && (!bending || !q)) || !(h > 0.f)) {
        ats::set_error("ats_energy_noalloc: need device arrays x, x_start, v, mass, fixed, out3, a host accel[3], "
                       "num_verts > 0, non-negative edge counts with their arrays, and h > 0");
        return ATS_ERR_INVALID;
    }
    if (num_verts > kNoallocMaxElements || num_edges > kNoallocMaxElements ||
        num_bending_edges > kNoallocMaxElements) {
        ats::set_error("ats_energy_noalloc: more than 8388608 vertices, edges or bending edges; the static scratch "
                       "holds 4096 partial sums of 2048 elements per term");
        return ATS_ERR_INVALID;
    }
    double* partials = nullptr;
    int r = partials_address(&partials);
    if (r) return r;
    const int nblk_v = (num_verts + kNoallocChunk - 1) / kNoallocChunk;
    const int nblk_e = (num_edges + kNoallocChunk - 1) / kNoallocChunk;
    const int nblk_b = (num_bending_edges + kNoallocChunk - 1) / kNoallocChunk;
    const int grid = nblk_v > nblk_e ? (nblk_v > nblk_b ? nblk_v : nblk_b) : (nblk_e > nblk_b ? nblk_e : nblk_b);
    NoallocArgs a;
    a.x = x;
    a.x_start = x_start;
    a.v = v;
    a.mass = mass;
    a.fixed = fixed;
    a.nv = num_verts;
    a.edges = edges;
    a.rest = rest_length;
    a.ne = num_edges;
    a.bending = bending;
    a.q = q;
    a.nb = num_bending_edges;
    a.k_stretch = k_stretch;
    a.k_bend = k_bend;
    a.ax = accel[0];
    a.ay = accel[1];
    a.az = accel[2];
    a.h = h;
    a.partials = partials;
    cudaStream_t st = (cudaStream_t)stream;
    energy_noalloc_kernel<<<grid, kNoallocThreads, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        energy_noalloc_final_kernel<<<1, kNoallocThreads, 0, st>>>(partials, nblk_v, nblk_e, nblk_b, out3);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        ats::set_error(std::string("ats_energy_noalloc: launch: ") + cudaGetErrorString(e));
        return ATS_ERR_CUDA;
    }
    return ATS_OK;
}
