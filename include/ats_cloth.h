/*
 * ats_cloth.h -- C ABI of the B200 cloth solver (libats_b200.so).
 *
 * The solver is the hot path of libAtsSim's cloth simulation: Vertex Block Descent
 * (inertial prediction, per-colour sweeps that gather mass-spring stretch and
 * quadratic bending gradients and 3x3 Hessians and solve a 3x3 block system, then
 * the velocity update) and XPBD per-colour constraint projection. Each entry point
 * below replaces one task of the reference's CPU/Metal implementation; the
 * function ids are those of src/heterogeneous/launcher.h (namespace Launcher).
 *
 * Conventions
 *   - Every call returns an int status: ATS_OK (0) or an ATS_ERR_* code; the
 *     message of the last failure on the calling thread is ats_last_error().
 *   - Handles own their device memory; one handle is used from one host thread.
 *   - `stream` is a cudaStream_t passed as a plain pointer (NULL = legacy default
 *     stream). Step entry points only enqueue work and return, like the Metal
 *     encode path of the reference (examples/example3_hybrid_cpu_gpu.cpp:1210-1377).
 *   - Host arrays are plain pointers; vertex arrays are in the caller's original
 *     vertex order, instances concatenated (instance 0 first).
 *   - There is no CPU fallback: without a usable CUDA device every compute call
 *     fails with ATS_ERR_CUDA.
 */
#ifndef ATS_CLOTH_H
#define ATS_CLOTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ATS_OK = 0,
    ATS_ERR_INVALID = 1,   /* bad argument (null pointer, out-of-range index, bad mesh) */
    ATS_ERR_CUDA = 2,      /* CUDA runtime error or no device */
    ATS_ERR_NOMEM = 3,     /* host or device allocation failed */
    ATS_ERR_TIMEOUT = 4,   /* a bounded device wait expired */
    ATS_ERR_STATE = 5      /* call not valid in the handle's current state */
};

enum { ATS_SOLVER_VBD = 0, ATS_SOLVER_XPBD = 1 };

/* Grid triangulation patterns for ats_grid_mesh. */
enum {
    ATS_GRID_UNIFORM = 0,    /* every quad split along (r,c)-(r+1,c+1) */
    ATS_GRID_ALTERNATING = 1 /* split alternates with (r+c) parity, the square40K.obj layout */
};

/* Which colouring / topology array to read back. */
enum {
    ATS_COLORING_VERTEX = 0,  /* VBD vertex colours (example2_async_iter.cpp:572-646) */
    ATS_COLORING_STRETCH = 1, /* XPBD edge colours (example2_async_iter.cpp:458-533) */
    ATS_COLORING_BENDING = 2  /* XPBD bending-edge colours (same function, nv = 4) */
};

typedef struct ats_topology ats_topology;
typedef struct ats_cloth ats_cloth;
typedef void* ats_stream;

/* One cloth instance. positions are the rest (and initial) state. */
typedef struct ats_instance_desc {
    int num_verts;
    const float* positions;      /* 3 * num_verts */
    int num_faces;
    const int* faces;            /* 3 * num_faces, 0-based, triangles */
    const float* mass;           /* num_verts, kg (SceneParams default_mass rules live in ats_mass_*) */
    const unsigned char* fixed;  /* num_verts, nonzero = pinned (sa_is_fixed) */
    float k_stretch;             /* stiffness_stretch_spring, N/m */
    float k_bend;                /* effective quadratic bending stiffness
                                    (SceneParams::get_stiffness_quadratic_bending()) */
} ats_instance_desc;

/* Solver parameters shared by all instances of a handle. */
typedef struct ats_solver_params {
    float implicit_dt;      /* frame step; the substep dt is implicit_dt / num_substep */
    int num_substep;        /* substeps per frame */
    int iterations;         /* constraint_iter_count */
    float damping;          /* damping_cloth: v *= exp(-damping * dt) */
    float gravity[3];       /* external acceleration, m/s^2 */
    int threads_per_vertex; /* VBD sweep lanes per vertex: 1, 2, 4 or 8; 0 = default (4) */
    int block_size;         /* VBD sweep threads per block (multiple of 32, <= 1024); 0 = default (128) */
} ats_solver_params;

typedef struct ats_cloth_info {
    int num_instances;
    int num_verts;          /* total over instances */
    int num_edges;
    int num_bending_edges;
    int num_vertex_colors;  /* max over instances */
    int num_stretch_colors;
    int num_bending_colors;
    int threads_per_vertex;
    int block_size;
    int stencil_slots;      /* stencil entries stored (incl. padding) */
    long long device_bytes; /* device memory held by the handle */
    int vbd_form;           /* fixed-iteration VBD iterations: 0 a launch per colour, 1 persistent */
    int xpbd_form;          /* XPBD iterations: 0 a launch per colour, 1 persistent */
    int list_form;          /* list sweep of residual-driven frames: 0 plain, 1 pipelined, 2 streamed */
    long long sweep_layout_bytes; /* bytes one VBD iteration of the streamed list sweep must move over
                                     every instance in this layout: the stencil rows as stored (8 B a
                                     slot, 4 more on edge rows), x read and written, x0 and vel per
                                     vertex, 28 B a slice (descriptor, metadata, list entry) */
    int tune_source;        /* shape and forms: 0 defaults or set explicitly, 1 timed by ats_autotune,
                               2 taken from the autotuning cache */
    int l2_persisting;      /* 1: list sweeps keep the positions in L2 as persisting lines */
} ats_cloth_info;

/* ---------------------------------------------------------------- host-only mesh helpers */

/* Regular n x n grid on y = 0 spanning [-0.5, 0.5]^2: vertex (r, c) -> r*n + c at
 * (-0.5 + c/(n-1), 0, -0.5 + r/(n-1)). positions: 3*n*n floats; faces: 6*(n-1)^2 ints. */
int ats_grid_mesh(int n, int pattern, float* positions, int* faces);

/* Pins of examples/example2_async_iter.cpp:195-209: AABB-normalised z < 0.01 and
 * (x > 0.99 or x < 0.01). */
int ats_reference_pins(const float* positions, int num_verts, unsigned char* fixed);

/* Area-lumped mass: each triangle gives a third of its area to each corner, scaled
 * so that the masses sum to total_mass. */
int ats_mass_area_weighted(const float* positions, int num_verts, const int* faces, int num_faces,
                           float total_mass, float* mass);

/* Reads the vertices and triangles of a Wavefront OBJ file (0-based faces,
 * degenerate triangles dropped as src/Utils/mesh_reader.cpp:170-177). Call with
 * null arrays first to get the counts. */
int ats_obj_read(const char* path, int* num_verts, float* positions, int* num_faces, int* faces);

/* Writes positions and triangles as an OBJ file ("v x y z", 1-based "f a b c"), as
 * src/Utils/mesh_reader.cpp:374-462 exports a simulated frame. */
int ats_obj_write(const char* path, const float* positions, int num_verts, const int* faces, int num_faces);
/* Cloth state (x, v, 3 floats per vertex) as a versioned little-endian file with an
 * FNV-1a checksum, for checkpoint / resume (replaces the raw dumps of
 * src/Utils/mesh_reader.h:323-343). Read with null x / v to get num_verts and frame;
 * otherwise *num_verts is the capacity on input and the count on output. */
int ats_state_write(const char* path, const float* x, const float* v, int num_verts, int frame);
int ats_state_read(const char* path, float* x, float* v, int* num_verts, int* frame);

/* ---------------------------------------------------------------- topology (host only)
 * Replaces SimMesh::extract_edges_from_surface (src/Utils/mesh_reader.h:206-298), the
 * adjacency set-up and greedy colourings of examples/example2_async_iter.cpp:229-304,
 * 442-697, and the rest state of :309-375. Integer results are bit-identical to the
 * reference algorithms. */
int ats_topology_build(const ats_instance_desc* mesh, ats_topology** out);
int ats_topology_destroy(ats_topology* topo);
/* counts[0..4] = edges, bending edges, vertex colours, stretch colours, bending colours */
int ats_topology_counts(const ats_topology* topo, int* counts);
int ats_topology_edges(const ats_topology* topo, int* edges /* 2E */, int* bending /* 4B */);
int ats_topology_rest(const ats_topology* topo, float* rest_length /* E */, float* q /* 16B, column-major */);
int ats_topology_coloring(const ats_topology* topo, int which, int* prefix /* C+1 */, int* items);

/* ---------------------------------------------------------------- solver handle */

/* Builds the topology of every instance, the colour-major device layout and uploads
 * it. Replaces CpuSolver::init_xpbd_system (example2_async_iter.cpp:442-697) for a
 * CUDA device. */
int ats_cloth_create(const ats_instance_desc* instances, int num_instances, const ats_solver_params* params,
                     ats_cloth** out);
int ats_cloth_destroy(ats_cloth* cloth);
int ats_cloth_query(const ats_cloth* cloth, ats_cloth_info* info);

/* Device order of the vertices: layout_of_caller[i] = position of caller vertex i in
 * the instance-major, colour-major device layout (recorded samples follow it). */
int ats_cloth_vertex_order(const ats_cloth* cloth, int* layout_of_caller);

/* Frame-end state (x, v), 3 floats per vertex, original order, instances concatenated.
 * Replaces SolverInterface::restart_system / load_saved_state and the frame_end read
 * (example2_async_iter.cpp:1575-1614). Both calls synchronise `stream`. v may be null. */
int ats_set_state(ats_cloth* cloth, const float* x, const float* v, ats_stream stream);
int ats_get_state(ats_cloth* cloth, float* x, float* v, ats_stream stream);
/* Current iterate x (mid-frame), same layout. Synchronises `stream`. */
int ats_get_positions(ats_cloth* cloth, float* x, ats_stream stream);
/* Replaces the current iterate x only (the frame start x0 and v stay). */
int ats_set_positions(ats_cloth* cloth, const float* x, ats_stream stream);

/* Per-instance external acceleration (gravity plus wind force / instance mass),
 * 3 floats per instance, read by the device at every predict / sweep; enqueued on
 * `stream` so that it takes effect for work queued after it. */
int ats_set_accel(ats_cloth* cloth, const float* accel, ats_stream stream);

/* --- step entry points (one per launcher task) --- */
/* id_xpbd_predict_position (launcher.h:92): x = x0 + h (v + h a), pinned: x = x0. */
int ats_predict_position(ats_cloth* cloth, ats_stream stream);
/* id_vbd_all_in_one (launcher.h:80) with cluster_idx = color: inertia + stretch +
 * bending gather and guarded 3x3 solve for every vertex of the colour. */
int ats_vbd_color_sweep(ats_cloth* cloth, int color, ats_stream stream);
/* `iterations` full VBD iterations (all colours in order), as
 * solve_constraints_VBD repeated (example2_async_iter.cpp:1481-1509). */
int ats_vbd_iterations(ats_cloth* cloth, int iterations, ats_stream stream);
/* id_xpbd_update_velocity (launcher.h:96): v = (x - x0)/h * exp(-damping h), x0 = x. */
int ats_update_velocity(ats_cloth* cloth, ats_stream stream);
/* id_xpbd_reset_constrains (launcher.h:93): lambda = 0. */
int ats_xpbd_reset_constraints(ats_cloth* cloth, ats_stream stream);
/* id_xpbd_constraint_stretch_mass_spring (launcher.h:21) for one colour. */
int ats_xpbd_stretch_color(ats_cloth* cloth, int color, ats_stream stream);
/* id_xpbd_constraint_bending (launcher.h:23) for one colour (quadratic bending). */
int ats_xpbd_bending_color(ats_cloth* cloth, int color, ats_stream stream);

/* One whole frame (substeps x (predict, iterations x colours, update)), as
 * CpuSolver::physics_step_vbd / physics_step_xpbd (example2_async_iter.cpp:1017-1143). */
int ats_frame(ats_cloth* cloth, int solver, ats_stream stream);
/* The same frame replayed from a CUDA graph captured on first use (per solver). */
int ats_frame_graph(ats_cloth* cloth, int solver, ats_stream stream);

/* One VBD frame iterated to a residual: predict, then VBD iterations in chunks of
 * `check_every`, after each chunk the FP64 residual of every instance; an instance
 * stops (its sweeps are skipped) once ||grad G(x)|| <= tol ||grad G(y)|| or after
 * max_iterations; then the velocity update. iterations / residual (host, one per
 * instance, nullable) receive the iterations used and the final relative residual.
 * The residual is the norm of the incremental-potential gradient over free vertices
 * relative to its value at y, the inertial prediction (the reference defines none);
 * the probes evaluate each vertex's gradient with the solver's FP32 force arithmetic
 * and sum in FP64 (ats_residual is FP64 throughout). The host reads the number of
 * active instances every fourth probe. */
int ats_frame_to_residual(ats_cloth* cloth, double tol, int check_every, int max_iterations, int* iterations,
                          double* residual, ats_stream stream);
/* The same with one tolerance per instance (host array) and, when first_check (host,
 * one per instance) is not null, a probe schedule per instance: instance i is probed
 * after first_check[i], first_check[i] + check_every, ... iterations and at
 * max_iterations (an instance whose iteration count is predictable, e.g. from its
 * previous frame, is probed once or twice instead of every check_every). */
int ats_frame_to_residuals(ats_cloth* cloth, const double* tols, const int* first_check, int check_every,
                           int max_iterations, int* iterations, double* residual, ats_stream stream);

/* Form of the iterations of fixed-iteration frames (and ats_vbd_iterations) for one
 * solver: 0 one launch per colour (the next colour's constant data loads while the
 * previous one drains); 1 persistent: all iterations in one cooperative launch, each
 * colour a grid-stride loop, a bounded grid barrier between colours. Both give the
 * same positions. A new handle starts with form 0 for both solvers; ats_autotune times
 * both forms and keeps the faster; this call overrides it (and drops captured frame
 * graphs). Fails with ATS_ERR_INVALID if the device cannot run form 1. The
 * residual-driven frames always use their persistent list sweep. */
int ats_set_sweep_form(ats_cloth* cloth, int solver, int form);

/* The sweep of the residual-driven frames (a resident grid striding over the slices of
 * the instances still iterating): 0 plain; 1 pipelined, where each warp stages its next
 * slice's stencil and vertex records in shared memory (cp.async) while it computes the
 * current one; 2 streamed, where the data read once per iteration (stencil, vertex
 * records, frame-start state) goes through evict-first loads, leaving L2 to the
 * positions, and each warp's next slice descriptor loads while the current slice
 * computes. Same positions. ats_autotune times the three and keeps the fastest. */
int ats_set_list_sweep(ats_cloth* cloth, int form);

/* on = 1: every list sweep of this handle keeps its positions in L2 as persisting lines
 * (an access-policy window over them on each launch), so that the neighbours the next
 * colours gather are still there after the colour's stencil has streamed past. While a
 * handle has it on, the context's persisting-L2 set-aside (cudaLimitPersistingL2CacheSize,
 * a per-context limit) is sized for its positions (up to the device maximum); the last
 * such handle to turn it off or be destroyed puts the previous size back. ATS_ERR_STATE
 * if the device has no persisting L2. Same positions. ats_autotune times it. */
int ats_set_l2_persisting(ats_cloth* cloth, int on);

/* Self-test of the bounded device waits, on the current device: one kernel waits at a
 * grid barrier (as the persistent kernels do) for arrivals that never come, one waits
 * on an mbarrier (as the tensor-core inference does) on which nothing arrives; each must
 * give up after `polls` polls and set its error word, and a kernel launched after them
 * must still run. Reports ATS_ERR_TIMEOUT in each status when its wait expired as
 * designed (ATS_OK if it did not), and returns ATS_ERR_STATE if the kernel after them
 * did not run. No fault or hang is involved: every wait is bounded. */
int ats_selftest_bounded_waits(unsigned polls, int* barrier_status, int* mbarrier_status);

/* Probe schedule of the residual-driven frames of this handle (ats_frame_to_residual(s),
 * ats_frame_warm_to_residual). 0 (default): every check_every iterations after an
 * instance's first probe, and at max_iterations. 1 (extrapolated): the first two probes
 * as policy 0; after that, from the residual's contraction per iteration between the
 * last two probes, the next probe comes after half of the iterations still predicted
 * to reach the tolerance (at least check_every, rounded up to a multiple of it), or at
 * max_iterations when the residual did not fall. Probes then follow the distance to the
 * tolerance instead of a fixed period; an instance can stop up to that gap after it
 * crossed the tolerance. The reference has no residual-driven frames. */
int ats_set_probe_policy(ats_cloth* cloth, int policy);

/* Times `iterations` VBD iterations (three times, taking the fastest) for every
 * lanes-per-vertex (1, 2, 4, 8) and block size (64, 128, 256) on this handle's own
 * mesh, keeps the fastest, then times the persistent form of the fixed-iteration VBD
 * and XPBD iterations (ats_set_sweep_form) and the forms of the list sweep
 * (ats_set_list_sweep) and keeps the fastest of each; reports the shape
 * (ats_cloth_query reports the forms). The iterate x is restored afterwards; captured frame graphs are dropped (they
 * are re-captured on next use). Synchronises `stream`. */
int ats_autotune(ats_cloth* cloth, int iterations, ats_stream stream, int* tpv, int* block_size);

/* The autotuning cache: ats_autotune records its choices (lanes per vertex, block size,
 * the three forms) per (GPU name and SM count, mesh class: vertex and instance counts in
 * power-of-two buckets, vertex, stretch and bending colour counts), and a later call on a
 * handle of the same GPU and class applies them without timing (ats_cloth_info's
 * tune_source = 2). The cache is per process; _save writes it as text ("ats-autotune 2",
 * then one "key tpv block vbd_form list_form xpbd_form l2_persisting" line per entry), _load merges
 * such a file (ATS_ERR_INVALID if it cannot be read or a line is malformed; nothing is merged
 * then), _clear empties it. No GPU is needed for these four. */
int ats_autotune_cache_size(void);
void ats_autotune_cache_clear(void);
int ats_autotune_cache_save(const char* path);
int ats_autotune_cache_load(const char* path);

/* Two-device asynchronous iteration, as example2_async_iter.cpp:1160-1200 and
 * example3 run it: both devices iterate on their own copy of the positions from a
 * common fork point, then the copies are merged.
 * ats_async_fork: the current iterate becomes the fork point (id_xpbd_copy_to_cpu_gpu,
 * example2_async_iter.cpp:1269-1273).
 * ats_async_merge: merges the other device's iterate (host, caller order, 3 floats per
 * vertex) into this handle's, as Core::read_and_solve_conflict
 * (xpbd_constraints.h:815-869) with this handle as "self": with weight > FLT_EPSILON,
 * fork + weight (dx_self + dx_other) where both moved, the one that moved otherwise;
 * else the average. The result is the new iterate and the new fork point.
 * Synchronises `stream`. */
int ats_async_fork(ats_cloth* cloth, ats_stream stream);
int ats_async_merge(ats_cloth* cloth, const float* other_positions, float weight, ats_stream stream);

/* FP64 incremental-potential energy of the current iterate against the current
 * frame start (Energy::compute_energy_* of xpbd_constraints.h:2079-2214):
 * out[0] = inertia, out[1] = stretch, out[2] = bending. Synchronises `stream`. */
int ats_energy(ats_cloth* cloth, double* out3, ats_stream stream);
/* FP64 norm of the incremental-potential gradient over free vertices, one value per
 * instance, of the current iterate (grad = m/h^2 (x - y) - f_stretch - f_bending,
 * y = x0 + h v + h^2 a). Synchronises `stream`. */
int ats_residual(ats_cloth* cloth, double* out_per_instance, ats_stream stream);
/* FP64 incremental potential G(x) per instance of the current iterate against the
 * current frame start: the three ats_energy terms of the instance, summed per vertex
 * over the merged neighbour stencil (the quantity the learned warm start's fallback
 * compares). Synchronises `stream`. */
int ats_potential(ats_cloth* cloth, double* out_per_instance, ats_stream stream);

/* FP64 energy of one cloth state given as plain device arrays, with no device
 * allocation. It has no counterpart in the reference. It is for callers that cannot
 * call cudaMalloc: programs whose GPU memory belongs to their own allocator (an
 * engine or framework that reserves the device heap up front), or per-frame loops
 * that cannot afford the device-wide synchronisation cudaMalloc / cudaFree may
 * cause. The caller passes device arrays in its own vertex order: x, x_start, v
 * (3 floats per vertex), mass, fixed (num_verts), edges (2 ints each) with
 * rest_length, bending (4 ints each) with q (16 floats each, column-major as
 * ats_topology_rest returns it); accel is 3 host floats, h the substep dt. out3
 * (device, 3 doubles) receives inertia, stretch and bending, the terms ats_energy
 * computes. Scratch is a static 96 KiB device array that every GPU which loads the
 * library keeps until exit: at most 8,388,608 vertices, edges and bending edges per
 * call (larger calls fail with ATS_ERR_INVALID). Every call looks up that array's
 * device address on the current device (a runtime query, no allocation); the first
 * call on a device may load the module, so make it before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and may return wrong
 * sums. Enqueues on `stream` and returns without synchronising. */
int ats_energy_noalloc(const float* x, const float* x_start, const float* v, const float* mass,
                       const unsigned char* fixed, int num_verts, const int* edges, const float* rest_length,
                       int num_edges, const int* bending, const float* q, int num_bending_edges, float k_stretch,
                       float k_bend, const float* accel, float h, double* out3, ats_stream stream);

/* ---------------------------------------------------------------- learned warm start
 * No counterpart in the reference: a per-vertex MLP (24 -> 64 -> 64 -> 64 -> 3, GELU
 * by a degree-8 polynomial within 1.2e-4 of z Phi(z) (csrc/ats_gelu.cuh, generated by
 * csrc/fit_gelu.py), BF16 weights and activations, FP32 accumulation on the tensor
 * cores) predicts
 * the frame's solved position; the plain VBD iterations always run afterwards.
 * Features of vertex v (h the substep, s = 9.8 h^2, y the inertial prediction):
 * h v / s, (y - x0) / s, and (x0_u - x0_v) / rest length of the edge neighbours in six
 * rest directions (+x, +x+z, +z, -x, -x-z, -z; zero where there is none). Output:
 * (x - y) / s; the guess is y + s * output, pinned vertices keep y. */
typedef struct ats_mlp ats_mlp;
typedef struct ats_dataset ats_dataset;

/* Parameter count (10115): FP32 master layout W1[24][64] b1[64] W2[64][64] b2 W3 b3
 * W4[64][3] b4[3], W[in][out] row-major. */
int ats_mlp_param_count(void);
int ats_mlp_create(unsigned long long seed, ats_mlp** out);
int ats_mlp_destroy(ats_mlp* mlp);
int ats_mlp_get_params(const ats_mlp* mlp, float* params);
/* Replaces the parameters and resets the optimiser state. */
int ats_mlp_set_params(ats_mlp* mlp, const float* params);
/* Input / output normalisation (54 floats): in_mean[24], in_scale[24] (1/std),
 * out_mean[3], out_std[3]; the network sees (f - in_mean) * in_scale and its raw
 * output o gives out_mean + out_std * o. A new model has the identity. */
int ats_mlp_get_normalization(const ats_mlp* mlp, float* norm);
int ats_mlp_set_normalization(ats_mlp* mlp, const float* norm);
/* Sets the normalisation from the FP64 column means / standard deviations of `data`. */
int ats_mlp_fit_normalization(ats_mlp* mlp, const ats_dataset* data, ats_stream stream);
/* Network outputs of n feature rows (24 floats each) into outputs (3 floats each),
 * normalisation applied. */
int ats_mlp_infer(const ats_mlp* mlp, const float* features, int n, float* outputs, ats_stream stream);
/* Gradient (FP32, ats_mlp_param_count floats) of the mean squared error over n
 * samples in normalised target space, and the loss; the parameters are not changed. */
int ats_mlp_gradient(ats_mlp* mlp, const float* features, const float* targets, int n, float* grad, float* loss,
                     ats_stream stream);

/* Training samples (features, targets) kept on the device. */
int ats_dataset_create(long long capacity, ats_dataset** out);
int ats_dataset_destroy(ats_dataset* data);
int ats_dataset_size(const ats_dataset* data, long long* n);
int ats_dataset_read(const ats_dataset* data, long long first, long long count, float* features, float* targets);
/* Records one frame of `cloth` as samples: call ats_record_frame_begin right after
 * ats_predict_position (features and y), run the iterations, then
 * ats_record_frame_end before ats_update_velocity (target (x - y)/s of every free vertex). */
int ats_record_frame_begin(ats_cloth* cloth, ats_stream stream);
int ats_record_frame_end(ats_cloth* cloth, ats_dataset* data, ats_stream stream);
/* Data-parallel training pieces: the gradient of one batch drawn from `data` (host
 * output, parameters unchanged), and one Adam step with a given gradient (for a
 * gradient averaged over ranks). Both synchronise `stream`. */
int ats_mlp_batch_gradient(ats_mlp* mlp, const ats_dataset* data, int batch, unsigned long long seed, float* grad,
                           float* loss, ats_stream stream);
int ats_mlp_apply_gradient(ats_mlp* mlp, const float* grad, float lr, ats_stream stream);
/* `steps` Adam steps on batches of `batch` samples drawn from `data` (seeded);
 * mean_loss (nullable) = mean loss of the last 20 steps. Synchronises `stream`. */
int ats_mlp_train(ats_mlp* mlp, const ats_dataset* data, int steps, int batch, float lr, unsigned long long seed,
                  float* mean_loss, ats_stream stream);
/* After ats_predict_position: x = learned guess. With fallback != 0 an instance keeps
 * y when its FP64 incremental potential G(guess) > G(y); used (host, one per instance,
 * nullable) receives 1 where the guess was kept (synchronises `stream` then). */
int ats_warm_start(ats_cloth* cloth, const ats_mlp* mlp, int fallback, int* used, ats_stream stream);
/* ats_frame with the learned guess between predict and the iterations; `iterations`
 * < 0 uses the handle's count. With use_graph != 0 the frame is replayed from a CUDA
 * graph captured on first use (re-captured when the model, count or fallback change;
 * the model's parameters may change between replays). */
int ats_frame_warm(ats_cloth* cloth, const ats_mlp* mlp, int fallback, int iterations, int use_graph,
                   ats_stream stream);
/* ats_frame_to_residuals with the learned guess; the residual stays relative to
 * ||grad G(y)|| of the inertial prediction. tols (host, one per instance) overrides tol when not null;
 * first_check (nullable) is the per-instance probe schedule of ats_frame_to_residuals. */
int ats_frame_warm_to_residual(ats_cloth* cloth, const ats_mlp* mlp, int fallback, double tol, const double* tols,
                               const int* first_check, int check_every, int max_iterations, int* iterations,
                               double* residual, int* used, ats_stream stream);

/* Kernels the library has launched in this process: every direct launch, plus the
 * kernel nodes of every CUDA-graph replay (a kernel enqueued during stream capture is
 * counted when its graph is replayed). A diagnostic with no counterpart in the
 * reference; benchmarks read it before and after a timed region. */
int ats_kernel_launches(long long* count);

/* Message of the last failed call on this thread ("" if none). */
const char* ats_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ATS_CLOTH_H */
