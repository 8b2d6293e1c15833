// ats_launcher.hpp -- the task / implementation / scheduler API of libAtsSim
// (src/heterogeneous/launcher.h, namespace Launcher) for Linux and CUDA.
//
// Same names, argument meanings and call order as the reference, so a solver
// written against launcher.h registers a CUDA implementation unchanged:
//
//   Launcher::Implementation gpu(Launcher::DeviceTypeGpu, [&](const Launcher::LaunchParam& p) { ... });
//   uint t = scheduler.add_task(Launcher::Task(Launcher::id_vbd_all_in_one, iter, -1u, color, {cpu, gpu}));
//   scheduler.set_connect(a, b);  scheduler.profile_from(...);
//   scheduler.topological_sort(); scheduler.standardizing_dag(); scheduler.scheduler_dag();
//   scheduler.launch(Launcher::Scheduler::LaunchModeGpu, task_to_param, false);
//
// Differences, all on the reference's Apple-only side: launch() works on Linux
// (the reference compiles its body only under __APPLE__, launcher.cpp:708-1581);
// the GPU "command list" is a CUDA stream; the Hetero mode runs the GPU tasks from a
// second host thread and orders CPU and GPU tasks with CUDA events and host counters
// (bounded waits) instead of MTLSharedEvent.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

namespace Launcher {

using uint = uint32_t;

// Task function ids, the full list of src/heterogeneous/launcher.h:14-221 in its order
// (so id_additional_root == 0 and the numeric values match the reference's), with
// TaskID_count last. Only the cloth-path ids have implementations in this library;
// the rest are names a caller's own tasks may carry.
#define ATS_LAUNCHER_FUNCTION_IDS(X) \
    X(id_additional_root) X(id_additional_terminal) X(id_task_heft_2002) \
    X(id_xpbd_constraint_stretch_mass_spring) X(id_xpbd_constraint_stretch_fem) X(id_xpbd_constraint_bending) \
    X(id_xpbd_constraint_stress) X(id_xpbd_constraint_inner_stress) X(id_xpbd_constraint_outer_stress) \
    X(id_xpbd_constraint_stretch_mass_spring_half) X(id_xpbd_constraint_stretch_fem_half) \
    X(id_xpbd_constraint_bending_half) X(id_xpbd_constraint_stress_half) X(id_xpbd_constraint_inner_stress_half) \
    X(id_xpbd_constraint_outer_stress_half) X(id_xpbd_constraint_self_collision_vv_addition_half) \
    X(id_xpbd_constraint_self_collision_vv_half) X(id_xpbd_constraint_self_collision_vv_half_cloth) \
    X(id_xpbd_constraint_self_collision_vv_half_tet) X(id_xpbd_constraint_self_collision_vv_half_cross) \
    X(id_xpbd_constraint_self_collision_vf_half) X(id_xpbd_constraint_self_collision_vv_addition) \
    X(id_xpbd_constraint_self_collision_vv) X(id_xpbd_constraint_self_collision_vv_cloth) \
    X(id_xpbd_constraint_self_collision_vv_tet) X(id_xpbd_constraint_self_collision_vv_cross) \
    X(id_xpbd_constraint_self_collision_vf) X(id_xpbd_constraint_obstacle_collision_vv) \
    X(id_xpbd_constraint_obstacle_collision_vv_cloth) X(id_xpbd_constraint_obstacle_collision_vv_tet) \
    X(id_xpbd_constraint_obstacle_collision_vf) X(id_xpbd_constraint_stretch_prev) \
    X(id_xpbd_constraint_stretch_post) X(id_xpbd_constraint_bending_prev) X(id_xpbd_constraint_bending_post) \
    X(id_xpbd_constraint_stress_prev) X(id_xpbd_constraint_stress_post) \
    X(id_xpbd_constraint_self_collision_prev) X(id_xpbd_constraint_self_collision_post) \
    X(id_xpbd_constraint_ground_collision) X(id_xpbd_constraint_ground_collision_cloth) \
    X(id_xpbd_constraint_ground_collision_tet) X(id_xpbd_constraint_ground_collision_stretch) \
    X(id_xpbd_constraint_ground_collision_bending) X(id_xpbd_constraint_ground_collision_self_collision) \
    X(id_xpbd_constraint_last_node) X(id_vbd_evaluate_inertia) X(id_vbd_evaluate_stretch_mass_spring) \
    X(id_vbd_evaluate_stretch_fem) X(id_vbd_evaluate_bending) X(id_vbd_evaluate_ground_collision) \
    X(id_vbd_evaluate_obstacle_collision) X(id_vbd_evaluate_self_collision) X(id_vbd_step) X(id_vbd_all_in_one) \
    X(id_sod_evaluate_energy_gauss_seidel) X(id_sod_evaluate_energy_hybrid) \
    X(id_sod_stretch_stencil_gauss_seidel) X(id_sod_stretch_stencil_hybrid) X(id_sod_init) X(id_sod_step) \
    X(id_sod_all_in_one) X(id_xpbd_predict_position) X(id_xpbd_reset_constrains) \
    X(id_xpbd_reset_collision_constrains) X(id_xpbd_store_previous_position) X(id_xpbd_update_velocity) \
    X(id_xpbd_copy_current_position_to_2_constraints) X(id_xpbd_copy_current_position_to_3_constraints) \
    X(id_xpbd_assemble_result_from_2_constraints) X(id_xpbd_assemble_result_from_3_constraints) \
    X(id_xpbd_copy_current_position_to_2_devices) X(id_xpbd_copy_current_position_to_constraints) \
    X(id_xpbd_assemble_result_from_constraints) X(id_xpbd_assemble_result_from_stretch_bending) \
    X(id_xpbd_assemble_result_from_stretch_collision) X(id_xpbd_assemble_result_from_bending_collision) \
    X(id_xpbd_assemble_result_from_stress_collision) X(id_xpbd_copy_to_stretch) X(id_xpbd_copy_to_bending) \
    X(id_xpbd_copy_to_self_collision_cloth) X(id_xpbd_copy_to_self_collision_tet) \
    X(id_xpbd_copy_to_sdf_collision_cloth) X(id_xpbd_copy_to_sdf_collision_tet) X(id_xpbd_copy_to_stress) \
    X(id_xpbd_get_from_stretch) X(id_xpbd_get_from_bending) X(id_xpbd_get_from_self_collision_cloth) \
    X(id_xpbd_get_from_self_collision_tet) X(id_xpbd_get_from_sdf_collision_cloth) \
    X(id_xpbd_get_from_sdf_collision_tet) X(id_xpbd_get_from_stress) X(id_xpbd_read_and_solve_conflict) \
    X(id_xpbd_copy_to_cpu_gpu) X(id_xpbd_get_from_cpu_gpu) X(id_xpbd_apply_constraint_delta_from_2_delta) \
    X(id_xpbd_sync_position_to_another_device) X(id_xpbd_update_cloth_position_from_2_devices) \
    X(id_xpbd_update_tet_position_from_2_devices) X(id_prepare_collision_detection_position) \
    X(id_update_global_aabb) X(id_self_collision_detection) X(id_self_collision_spatial_hashing_update) \
    X(id_self_collision_reset_collision_system_and_spatial_hashing) \
    X(id_self_collision_reset_collision_system_and_lbvh) X(id_self_collision_fill_in_hash_table) \
    X(id_self_collision_scan_hash_table) X(id_self_collision_insert_vert_into_hash_table) \
    X(id_self_collision_spatial_hashing_query) X(id_self_collision_narrow_phase_vv) \
    X(id_self_collision_narrow_phase_vf) X(id_self_collision_scan_and_fill_in_vv) \
    X(id_self_collision_scan_and_fill_in_vf) X(id_obstacle_collision_detection) \
    X(id_obstacle_collision_spatial_hashing_update) \
    X(id_obstacle_collision_reset_collision_system_and_spatial_hashing) \
    X(id_obstacle_collision_reset_collision_system_and_lbvh) X(id_obstacle_collision_fill_in_hash_table) \
    X(id_obstacle_collision_scan_hash_table) X(id_obstacle_collision_insert_vert_into_hash_table) \
    X(id_obstacle_collision_spatial_hashing_query) X(id_obstacle_collision_narrow_phase_vv) \
    X(id_obstacle_collision_narrow_phase_vf) X(id_obstacle_collision_scan_and_fill_in_vv) \
    X(id_obstacle_collision_scan_and_fill_in_vf) X(id_self_collision_compute_vert_aabb_and_center) \
    X(id_self_collision_compute_face_aabb_and_center) X(id_self_collision_compute_morton) \
    X(id_self_collision_init_tree) X(id_self_collision_sort_by_morton) X(id_self_collision_apply_sorted_morton) \
    X(id_self_collision_construct_tree_karras2012) X(id_self_collision_check_healthy) \
    X(id_self_collision_compute_escape_index) X(id_self_collision_compute_left_index) \
    X(id_self_collision_update_vert_aabb_dcd) X(id_self_collision_update_face_aabb_dcd) \
    X(id_self_collision_apply_leaves_aabb) X(id_self_collision_reset_lbvh) \
    X(id_self_collision_query_from_cloth_vert) X(id_obstacle_collision_compute_vert_aabb_and_center) \
    X(id_obstacle_collision_compute_face_aabb_and_center) X(id_obstacle_collision_compute_morton) \
    X(id_obstacle_collision_init_tree) X(id_obstacle_collision_sort_by_morton) \
    X(id_obstacle_collision_apply_sorted_morton) X(id_obstacle_collision_construct_tree_karras2012) \
    X(id_obstacle_collision_check_healthy) X(id_obstacle_collision_compute_escape_index) \
    X(id_obstacle_collision_compute_left_index) X(id_obstacle_collision_update_vert_aabb_dcd) \
    X(id_obstacle_collision_update_face_aabb_dcd) X(id_obstacle_collision_apply_leaves_aabb) \
    X(id_obstacle_collision_reset_lbvh) X(id_obstacle_collision_query_from_cloth_vert) \
    X(id_graph_coloring_vivace_vv) X(id_graph_coloring_vivace_vv_cloth) X(id_graph_coloring_vivace_vv_tet) \
    X(id_graph_coloring_vivace_vv_cross) X(id_graph_coloring_vivace_vv_wait_for_num_color) \
    X(id_graph_coloring_vivace_vf) X(id_reduce_degree_and_set_max_color_from_max_degree_vv) \
    X(id_reduce_degree_and_set_max_color_from_max_degree_vf) X(id_scan_uncolored_set) X(id_init_palette) \
    X(id_random_coloring_loops_vv) X(id_random_coloring_loops_vf) X(id_tentative_coloring) \
    X(id_conflict_resolution_vv) X(id_conflict_resolution_vf) X(id_feed_hungry_and_make_indirect_buffer) \
    X(id_put_rest_vertices_into_additional_color) X(id_put_rest_vertices_into_random_color) \
    X(id_make_cluster_indirect_cmd_buffer) X(id_xpbd_non)

enum FunctionID : uint {
#define ATS_LAUNCHER_ENUM_ENTRY(name) name,
    ATS_LAUNCHER_FUNCTION_IDS(ATS_LAUNCHER_ENUM_ENTRY)
#undef ATS_LAUNCHER_ENUM_ENTRY
    TaskID_count
};

// Printable name of every id (launcher.h:223-426).
extern const std::unordered_map<FunctionID, std::string> taskNames;

struct LaunchParam {
    FunctionID function_id = id_xpbd_non;
    uint startIdx = 0;
    uint endIdx = 1;
    uint blockDim = 256;
    uint queue_idx = 0;
    uint fence_idx = 0;
    uint iter_idx = 0;
    uint cluster_idx = 0;
    bool launch_indirect = false;
    bool test_time = false;
    bool use_hetero = false;
    bool is_allocated_to_main_device = true;
    uint buffer_idx = 0;
    uint left_buffer_idx = -1u;
    uint right_buffer_idx = -1u;
    std::vector<uint> input_buffer_idxs;
    std::vector<uint> output_buffer_idxs;
    uint get_thread_num() const { return endIdx - startIdx; }
};

using DeviceType = uint;
const DeviceType DeviceTypeCpu = 0;
const DeviceType DeviceTypeGpu = 1;
const DeviceType DeviceType0 = 0;
const DeviceType DeviceType1 = 1;
const DeviceType DeviceType2 = 2;

struct Implementation {
    DeviceType device = DeviceTypeCpu;
    std::function<void(const LaunchParam&)> implementation;
    Implementation() : implementation([](const LaunchParam&) {}) {}
    Implementation(const DeviceType& d, const std::function<void(const LaunchParam&)>& fn) : device(d), implementation(fn) {}
    void launch_task(const LaunchParam& p) const { implementation(p); }
    bool operator==(const Implementation& r) const { return device == r.device; }
};

struct Task {
    FunctionID func_id = id_xpbd_non;
    uint num_threads = 0;
    uint start_idx = 0;
    uint block_dim = 256;
    uint iter_idx = -1u;
    uint constraint_idx = -1u;
    uint cluster_idx = 0;
    bool can_be_seperate = false;
    bool is_num_threads_constant = true;
    bool is_computation_time_constant = false;  // excluded from the runtime refit of its cost
    bool is_memory_only_pass = false;
    bool use_indirect_dispatch = false;
    bool is_empty_node = false;
    std::vector<Implementation> list_implementation;
    // asynchronous-iteration buffer assignment (left / right neighbour buffers, the
    // task's own buffer and the other device's inputs) and the tasks behind them
    uint buffer_left = -1u, task_left = -1u;
    uint buffer_right = -1u, task_right = -1u;
    uint buffer_out = -1u, task_out = -1u;
    uint buffer_idx = -1u;
    bool is_allocated_to_main_device = true;
    bool is_first_iterative_task = false;
    std::vector<uint> buffer_ins, buffer_outs, buffer_idxs;
    std::vector<uint> task_ins, task_outs, task_idxs;
    std::vector<uint> resources;     // resource ids the task touches (caller-defined)
    std::vector<uint> predecessors;  // tasks this one waits for
    std::vector<uint> successors;    // tasks waiting for this one
    std::vector<float> list_weight;  // edge weight per successor

    Task() = default;
    Task(const FunctionID& f, const uint& numThreads, const bool& canBeSeparate, const bool& isNumThreadsConstant,
         const std::vector<Implementation>& imps)
        : func_id(f), num_threads(numThreads), can_be_seperate(canBeSeparate),
          is_num_threads_constant(isNumThreadsConstant), list_implementation(imps) {}
    Task(const FunctionID& f, const uint& clusterIdx, const std::vector<Implementation>& imps)
        : func_id(f), cluster_idx(clusterIdx), list_implementation(imps) {}
    Task(const FunctionID& f, const uint& iterIdx, const uint& constraintIdx, const uint& clusterIdx,
         const std::vector<Implementation>& imps)
        : func_id(f), iter_idx(iterIdx), constraint_idx(constraintIdx), cluster_idx(clusterIdx), list_implementation(imps) {}
    Task(const FunctionID& f, const uint& iterIdx, const uint& constraintIdx, const uint& clusterIdx,
         const std::vector<uint>& taskResources, const std::vector<Implementation>& imps)
        : func_id(f), iter_idx(iterIdx), constraint_idx(constraintIdx), cluster_idx(clusterIdx),
          list_implementation(imps), resources(taskResources) {}

    void add_front(const uint& i) { successors.push_back(i); }
    void add_back(const uint& i) { predecessors.push_back(i); }
    bool has_implementation(const DeviceType& t) const;
    // The implementation for device `t`; sets find and falls back to the first one.
    const Implementation& get_implementation(const DeviceType& t, bool& find) const;
    // "Task <tid> in iteration <i>'s cluster <c> => <name>" on stdout.
    void print_with_cluster(const uint tid) const;
};

// One scheduled task: processor and [start, end) in cost units.
struct ScheduleEvent {
    uint task_id = 0;
    uint proc = 0;
    float start = 0.f;
    float end = 0.f;
    ScheduleEvent() = default;
    ScheduleEvent(uint t, uint p, float s, float e) : task_id(t), proc(p), start(s), end(e) {}
    bool operator<(const ScheduleEvent& r) const { return end != r.end ? end < r.end : start < r.start; }
};

// A cross-device wait: task `task_id` on `proc` must not start before `wait_task`
// (on the other processor) has finished.
struct WaitEvent {
    uint task_id;
    uint proc;
    uint wait_task;
};

// A run of consecutive scheduled tasks on one processor, proc_schedules[proc]
// [start_idx, end_idx]: only its first task waits for the other processor and only
// its last one is waited for (the reference's launch events, one command buffer each
// on the GPU). waits: the other processor's tasks it depends on; signal: whether a
// task on the other processor depends on it.
struct LaunchEvent {
    uint proc = 0;
    uint start_idx = 0;
    uint end_idx = 0;
    std::vector<uint> waits;
    bool signal = false;
};

// Status of the last launch() (get_last_launch_status).
enum LaunchStatus { LaunchOk = 0, LaunchWaitTimeout = 1, LaunchMissingImplementation = 2, LaunchCudaError = 3,
                    LaunchTaskFailed = 4 };

const float inf = 99999.0f;
const uint input_buffer_mask = 0x0FFFFFFF;

class Scheduler {
public:
    enum LaunchMode {
        LaunchModeCpu,               // every task on its CPU implementation, scheduled / topological order
        LaunchModeGpu,               // every task on its GPU implementation (CPU where there is none)
        LaunchModePartialCPU,        // only the scheduled tasks allocated to processor 0
        LaunchModePartialGPU,        // only the scheduled tasks allocated to processor 1
        LaunchModeHetero,            // the HEFT schedule on CPU + GPU at once: GPU tasks from a second host
                                     // thread, cross-device order by CUDA events and host counters
        LaunchModeProgressiveHetero, // same as Hetero here (no command-buffer limit on CUDA)
        LaunchModeFakeHetero,        // the schedule, each task on its allocated device, synchronously
        LaunchModeSequeceHetero,     // the schedule, every task on the CPU implementation
    };

    Scheduler() = default;

    uint add_task(const Task& task);
    Task& get_task_by_tid(const uint& tid) { return list_task[tid]; }
    uint find_task_by_func_id(const FunctionID id) const;
    void set_connect(const uint& a, const uint& b, const float& weight = 1.0f);
    float delete_connect(const uint& a, const uint& b);
    void set_constraint_task_orders(const std::vector<uint>& orders) { constraint_task_orders = orders; }

    const std::vector<Task>& get_list_task() const { return list_task; }
    const std::vector<uint>& get_list_order() const { return list_order; }
    const std::vector<uint>& get_sorted_nodes() const { return sorted_nodes; }
    const std::vector<ScheduleEvent>& get_task_schedules() const { return task_schedules; }
    const std::vector<std::vector<ScheduleEvent>>& get_proc_schedules() const { return proc_schedules; }
    const std::vector<double>& get_ranku() const { return ranku; }
    const std::vector<WaitEvent>& get_wait_events() const { return wait_events; }
    const std::vector<std::vector<LaunchEvent>>& get_launch_events() const { return launch_events; }

    // Depth-first topological order; false (and an empty order) if the graph has a cycle.
    bool topological_sort();
    // Measured costs: `repeats` launches of one representative task per distinct
    // (function id, cluster) on every processor 0..nprocs-1 that implements it, in
    // milliseconds; processors without an implementation get `inf`. A processor with a
    // stream (set_device_stream) is timed by CUDA events recorded on that stream around
    // the launches, the CPU by the host clock. The result feeds profile_from, as the
    // reference's evaluate_compuatation_matrix feeds it (example3:1989-2316).
    void profile_costs(const std::function<LaunchParam(const Task&)>& task_to_param, int repeats, uint nprocs,
                       std::vector<std::pair<FunctionID, uint>>& keys, std::vector<std::vector<double>>& costs);
    // Costs per (function id, cluster) -> per-processor cost (launcher.cpp:645-704).
    void profile_from(const std::vector<std::pair<FunctionID, uint>>& map_tasks,
                      const std::vector<std::vector<double>>& map_costs, std::vector<double>& cost_total);
    // Adds a zero-cost root before every source and a terminal after every sink.
    void standardizing_dag(const std::vector<std::function<void(const LaunchParam&)>>& empty_fns = {});
    // HEFT: upward rank, then earliest-finish-time insertion on every processor.
    void scheduler_dag();
    // Cross-device waits of the schedule (two processors) and the launch events built
    // from them.
    void make_wait_events();
    // Runs the tasks; task_to_param builds the LaunchParam of a task.
    void launch(LaunchMode mode, const std::function<LaunchParam(const Task&)>& task_to_param, bool fully_not_wait,
                const std::vector<std::function<void()>>& assemble_impl = {});

    float fn_get_communication_cost(uint proc, uint pred_node, uint node) const;
    float fn_get_inner_communication_cost(uint proc) const;
    float get_scheduled_end_time() const;
    std::vector<float> get_scheduled_speedups() const;
    void print_proc_schedules() const;
    void print_speedups_to_each_device() const;
    void print_sort_by_typology() const;
    // The schedule as plottable lists (launcher.cpp:3915): per processor
    // "(colour key, task, buffer, start, end)" tuples, the colour key being a per
    // function-id base plus the cluster; then the cross-device dependencies as
    // "(pred proc, pred task, proc, task, pred end, start)". Reports tasks whose
    // scheduled length differs from the computation matrix.
    void print_schedule_to_graph_xpbd() const;
    void set_print_scheduling_datail(const bool b) { print_detail = b; }
    void set_safety_check(const bool b) { safety_check = b; }
    // How to drain a device queue before a host task or at the end of launch();
    // the GPU default synchronises the device stream (set_device_stream), else the
    // current CUDA device.
    void set_device_sync(DeviceType d, std::function<void()> fn);
    // The cudaStream_t on which the device's implementations enqueue their work
    // (passed as a pointer): Hetero launches record their completion events on it and
    // profile_costs times it with CUDA events.
    void set_device_stream(DeviceType d, void* cuda_stream);
    // Upper bound of every host-side wait of a Hetero launch (for a GPU task to
    // complete, for the other thread to reach a point); default 10 s. A wait that runs
    // out ends the launch with LaunchWaitTimeout instead of hanging.
    void set_wait_timeout_ms(double ms) { wait_timeout_ms = ms; }
    LaunchStatus get_last_launch_status() const { return last_status; }
    // After every Hetero launch, move the computation matrix toward the measured run
    // (launcher.cpp:711-793): per launch event, the difference between its measured
    // time and the sum of its tasks' costs (plus the inner communication cost between
    // consecutive tasks) is shared equally by its tasks whose
    // is_computation_time_constant is false, and each such cost becomes
    // max(cost + share / 2, 0). On by default.
    void set_runtime_refit(bool b) { runtime_refit = b; }
    // The refit itself, given the measured milliseconds of every launch event of
    // processor 0 and processor 1 (public so that a caller can refit from its own
    // timings).
    void refit_runtime_cost(const std::vector<float>& runtime_cost_cpu, const std::vector<float>& runtime_cost_gpu);
    // Measured milliseconds of the launch events of the last Hetero launch, per
    // processor (GPU events by CUDA events, CPU events by the host clock).
    const std::vector<std::vector<float>>& get_last_runtime_costs() const { return last_runtime_costs; }

public:
    std::vector<std::vector<float>> computation_matrix;  // [task][proc]
    std::vector<double> summary_of_costs_each_device;
    // diagonal: cost inside one device; off-diagonal: transfer speed (weight / speed)
    std::vector<std::vector<float>> communication_speed_matrix = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
    // constant per-pair delay used instead of weight / speed when non-empty
    std::vector<std::vector<float>> communication_cost_matrix_uma = {{0.002f, 0.220f}, {0.145f, 0.01f}};
    std::vector<float> communication_startup = {0, 0, 0};  // one entry per processor
    uint root_node = -1u, terminal_node = -1u;

private:
    void launch_hetero(const std::function<LaunchParam(const Task&)>& task_to_param, bool fully_not_wait);
    void compute_ranku(uint num_procs);
    double avg_cost(uint tid, uint num_procs) const;
    ScheduleEvent compute_eft(uint node, uint proc) const;
    void drain(DeviceType d) const;

    std::vector<Task> list_task;
    std::vector<uint> list_order;
    std::vector<uint> sorted_nodes;
    std::vector<uint> constraint_task_orders;
    std::vector<double> ranku;
    std::vector<std::vector<double>> avg_weight;
    std::vector<ScheduleEvent> task_schedules;
    std::vector<std::vector<ScheduleEvent>> proc_schedules;
    std::vector<WaitEvent> wait_events;
    std::vector<std::vector<LaunchEvent>> launch_events;
    std::vector<std::vector<float>> last_runtime_costs;
    std::map<DeviceType, std::function<void()>> device_sync;
    std::map<DeviceType, void*> device_stream;
    double wait_timeout_ms = 10000.0;
    LaunchStatus last_status = LaunchOk;
    bool runtime_refit = true;
    bool print_detail = false;
    bool safety_check = true;
};

}  // namespace Launcher
