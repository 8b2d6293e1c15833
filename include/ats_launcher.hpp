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
// the GPU "command list" is a CUDA stream drained with a device-sync hook; the
// Hetero mode orders CPU and GPU tasks with CUDA events instead of MTLSharedEvent.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace Launcher {

using uint = uint32_t;

// Task function ids used by the cloth path and the scheduler (launcher.h:14-221).
enum FunctionID : uint {
    id_xpbd_non = 0,
    id_additional_root,
    id_additional_terminal,
    id_task_heft_2002,
    id_xpbd_constraint_stretch_mass_spring,
    id_xpbd_constraint_bending,
    id_xpbd_constraint_last_node,
    id_xpbd_constraint_self_collision_vv_half_cloth,
    id_vbd_evaluate_inertia,
    id_vbd_evaluate_stretch_mass_spring,
    id_vbd_evaluate_bending,
    id_vbd_step,
    id_vbd_all_in_one,
    id_xpbd_predict_position,
    id_xpbd_reset_constrains,
    id_xpbd_reset_collision_constrains,
    id_xpbd_update_velocity,
    id_xpbd_copy_to_cpu_gpu,
    id_xpbd_read_and_solve_conflict,
    id_count
};

extern const std::map<FunctionID, std::string> taskNames;

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
    bool is_empty_node = false;
    std::vector<Implementation> list_implementation;
    // async-iteration buffer assignment (filled by a scheduler that assigns buffers)
    uint buffer_left = -1u, buffer_right = -1u, buffer_out = -1u, buffer_idx = -1u;
    bool is_allocated_to_main_device = true;
    std::vector<uint> buffer_ins, buffer_outs;
    std::vector<uint> resources;
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

    void add_front(const uint& i) { successors.push_back(i); }
    void add_back(const uint& i) { predecessors.push_back(i); }
    bool has_implementation(const DeviceType& t) const;
    // The implementation for device `t`; sets find and falls back to the first one.
    const Implementation& get_implementation(const DeviceType& t, bool& find) const;
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

const float inf = 99999.0f;
const uint input_buffer_mask = 0x0FFFFFFF;

class Scheduler {
public:
    enum LaunchMode {
        LaunchModeCpu,               // every task on its CPU implementation, scheduled / topological order
        LaunchModeGpu,               // every task on its GPU implementation (CPU where there is none)
        LaunchModePartialCPU,        // only the scheduled tasks allocated to processor 0
        LaunchModePartialGPU,        // only the scheduled tasks allocated to processor 1
        LaunchModeHetero,            // the HEFT schedule on CPU + GPU, ordered by CUDA events
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

    // Depth-first topological order; false (and an empty order) if the graph has a cycle.
    bool topological_sort();
    // Measured costs: `repeats` launches of one representative task per distinct
    // (function id, cluster) on every processor 0..nprocs-1 that implements it, each
    // followed by the device drain, host-timed in milliseconds; processors without an
    // implementation get `inf`. The result feeds profile_from (the reference refits
    // its matrix from command-buffer timestamps, launcher.cpp:711-793).
    void profile_costs(const std::function<LaunchParam(const Task&)>& task_to_param, int repeats, uint nprocs,
                       std::vector<std::pair<FunctionID, uint>>& keys, std::vector<std::vector<double>>& costs);
    // Costs per (function id, cluster) -> per-processor cost (launcher.cpp:645-704).
    void profile_from(const std::vector<std::pair<FunctionID, uint>>& map_tasks,
                      const std::vector<std::vector<double>>& map_costs, std::vector<double>& cost_total);
    // Adds a zero-cost root before every source and a terminal after every sink.
    void standardizing_dag(const std::vector<std::function<void(const LaunchParam&)>>& empty_fns = {});
    // HEFT: upward rank, then earliest-finish-time insertion on every processor.
    void scheduler_dag();
    // Cross-device waits of the schedule (two processors).
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
    void set_print_scheduling_datail(const bool b) { print_detail = b; }
    void set_safety_check(const bool b) { safety_check = b; }
    // How to drain a device queue before a host task or at the end of launch();
    // the GPU default synchronises the current CUDA device.
    void set_device_sync(DeviceType d, std::function<void()> fn);

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
    std::map<DeviceType, std::function<void()>> device_sync;
    bool print_detail = false;
    bool safety_check = true;
};

}  // namespace Launcher
