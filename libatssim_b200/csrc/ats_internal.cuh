// ats_internal.cuh -- handle layout and helpers shared by the library's .cu files.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/ats_cloth.h"
#include "ats_topology.hpp"

namespace ats {

void set_error(const std::string& msg);

#define ATS_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess) {                                                                \
            set_error(std::string(#call) + ": " + cudaGetErrorString(_e));                      \
            return ATS_ERR_CUDA;                                                                \
        }                                                                                       \
    } while (0)

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc((void**)&p, count * sizeof(T));
    }
    size_t bytes() const { return n * sizeof(T); }
};

inline cudaStream_t S(ats_stream s) { return (cudaStream_t)s; }

// Kernel-launch accounting behind ats_kernel_launches: count_launch after every direct
// launch (skipped while `st` is being captured, since the kernel then becomes a graph
// node), register_graph when a graph is instantiated (its kernel nodes are counted
// once), count_graph_launch at every replay.
void count_launch(cudaStream_t st);
void register_graph(cudaGraphExec_t exec, cudaGraph_t g);
void count_graph_launch(cudaGraphExec_t exec);

}  // namespace ats

struct ats_cloth {
    using Layout = ats::Layout;
    template <typename T>
    using DevBuf = ats::DevBuf<T>;
    Layout L;
    ats_solver_params prm{};
    int device = 0;
    int block = 128;
    float h = 0.f, h2inv = 0.f, damp = 1.f;
    // device arrays
    DevBuf<float4> x, x0, vel, vm, inst;
    DevBuf<int2> st_iw;
    DevBuf<float> st_rest;
    DevBuf<int4> slices;
    DevBuf<int> slice_inst;     // instance of each slice
    DevBuf<int2> slice_meta;    // per slice {instance, bit k = vertex k of the slice pinned}
    DevBuf<int> color_slices;   // n_vcolors + 1 slice offsets per colour
    DevBuf<int> act_list, act_count;  // per colour, the slices of instances still iterating
    DevBuf<int2> xs_edge;
    DevBuf<float> xs_rest, xs_k, xs_lambda;
    DevBuf<int4> xb_idx;
    DevBuf<float4> xb_q;
    DevBuf<float> xb_lambda;
    DevBuf<int> xs_color_d, xb_color_d;  // XPBD colour offsets, for the persistent kernel
    DevBuf<unsigned> loop_bar;           // its grid barrier: arrivals since the launch, bit 31 error
    DevBuf<int> loop_err;                // set when a barrier wait ran out
    int xpbd_loop_capable = 0;           // co-resident blocks of the persistent XPBD kernel (0: unavailable)
    int xpbd_loop_blocks = 0;            // the blocks XPBD frames launch it with (0: per-colour launches)
    int vbd_loop_blocks = 0;             // the same for VBD iterations (0: one launch per colour; set by autotune)
    int list_form = 0;                   // list sweep of residual-driven frames: 0 plain, 1 pipelined, 2 streamed
    int tune_source = 0;                 // shape and forms: 0 defaults or explicit, 1 timed, 2 tuning cache
    bool l2_keep = false;                // list sweeps keep the positions persisting in L2
    cudaAccessPolicyWindow l2_window{};  // their access-policy window (empty when off)
    DevBuf<int2> en_edge;
    DevBuf<float> en_rest, en_k, en_q, en_kb;
    DevBuf<int4> en_bend;
    DevBuf<int> inst_seg;
    DevBuf<int> to_caller;
    DevBuf<float> io_x, io_v;  // caller-order staging of the state
    DevBuf<float4> async_begin;  // fork point of two-device asynchronous iteration
    // scratch of the FP64 reductions
    DevBuf<double> partial, seg_partial, red_out, g2, norm0, tols;
    DevBuf<int> active, iters, n_active, due, first_check;  // ats_frame_to_residual bookkeeping
    DevBuf<int> next_due, last_it;                          // its extrapolated probe schedule
    DevBuf<double> last_res;
    int probe_policy = 0;                                   // 0 fixed, 1 extrapolated (ats_set_probe_policy)
    DevBuf<int> probe_points, probe_idx;                     // its probe schedule, on the device
    std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> chunk_graphs;  // residual-frame pieces
    int* host_flag = nullptr;             // pinned copy of n_active
    // learned warm start (uploaded at create; the rest allocated on first use)
    DevBuf<int> feat_nb, inst_eseg, inst_bseg, free_list;
    DevBuf<float> feat_len, feat_stage;
    DevBuf<float4> y_buf;
    DevBuf<double> pot_y, pot_guess, pot_vx, pot_vy;
    DevBuf<int> guess_used;
    DevBuf<int> tc_err;  // set by the tensor-core inference kernel when a completion wait ran out
    cudaGraphExec_t warm_graph = nullptr;  // captured warm-started frame (ats_frame_warm)
    const void* warm_key_mlp = nullptr;
    int warm_key_iters = -1, warm_key_fallback = -1;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};

    void drop_graphs() {
        for (auto& g : graph)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        if (warm_graph) {
            cudaGraphExecDestroy(warm_graph);
            warm_graph = nullptr;
        }
        for (auto& kv : chunk_graphs) cudaGraphExecDestroy(kv.second);
        chunk_graphs.clear();
    }
    ~ats_cloth() {
        drop_graphs();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        if (host_flag) cudaFreeHost(host_flag);
    }
    size_t device_bytes() const {
        return x.bytes() + x0.bytes() + vel.bytes() + vm.bytes() + inst.bytes() + st_iw.bytes() + st_rest.bytes() +
               slices.bytes() + slice_inst.bytes() + slice_meta.bytes() + color_slices.bytes() + act_list.bytes() + act_count.bytes() + xs_edge.bytes() + xs_rest.bytes() + xs_k.bytes() + xs_lambda.bytes() +
               xb_idx.bytes() + xb_q.bytes() + xb_lambda.bytes() + en_edge.bytes() + en_rest.bytes() + en_k.bytes() +
               en_q.bytes() + en_kb.bytes() + en_bend.bytes() + inst_seg.bytes() + to_caller.bytes() + io_x.bytes() +
               io_v.bytes() + async_begin.bytes() + partial.bytes() +
               seg_partial.bytes() + red_out.bytes() + g2.bytes() + norm0.bytes() + active.bytes() + iters.bytes() +
               n_active.bytes();
    }
};


namespace ats {

// Kernel launches of one handle (ats_cloth.cu); each returns an ATS_* status.
int launch_predict(ats_cloth* c, cudaStream_t st);
int launch_update(ats_cloth* c, cudaStream_t st);
// With `active` (the residual-driven frames' flags), a sweep runs over the per-colour
// lists of active slices that enqueue_compaction built from those flags.
int launch_sweep(ats_cloth* c, int color, cudaStream_t st, const int* active = nullptr);
int enqueue_iterations(ats_cloth* c, int solver, int iterations, cudaStream_t st, const int* active = nullptr);
// ||grad G|| per instance into c->red_out.p (FP64 throughout, or FP32 per-vertex terms
// with FP64 sums); with `active`, instances whose flag is 0 keep their previous values
int enqueue_residual_norms(ats_cloth* c, cudaStream_t st, const int* active = nullptr, bool fp32_terms = false);
// Per instance, the FP64 incremental potential G of the current positions (gx) and of
// y (gy), both against the inertial prediction y (ninst values each, device pointers).
int enqueue_potential_pair(ats_cloth* c, const float4* y, double* gx, double* gy, cudaStream_t st);
// Per instance, G(x) against the inertial prediction of the current frame start.
int enqueue_potential(ats_cloth* c, double* g, cudaStream_t st);
// ats_frame_to_residual(s) with an optional hook run after ||grad G(y)|| is taken and
// before the first iteration (the learned warm start replaces y there). Probes use
// FP32 per-vertex gradient terms and FP64 sums. first_check (host, per instance,
// nullable) = iteration of an instance's first probe.
int frame_to_residual_impl(ats_cloth* c, double tol, const double* tols, const int* first_check, int check_every,
                           int max_iterations, int* iterations, double* residual, cudaStream_t st,
                           const std::function<int(cudaStream_t)>& after_predict);

}  // namespace ats
