// The scheduler call sequence of CpuSolver::physics_step_vbd_async
// (examples/example2_async_iter.cpp:1305-1460), written the way that example writes it,
// against include/ats_launcher.hpp: task registration with the reference's Task
// constructors (including the one with a resource list), the per-cluster chaining of
// iterations, constraint task orders, profile_from with a constant cost list, the UMA
// communication matrix, topological sort, standardisation, HEFT, the schedule print
// calls, wait events, a designated-initialiser task_to_param and a launch.
//
// The implementations only record which task ran where; the program prints one JSON
// line: the launch order (function id, iteration, cluster), the device of each run, the
// scheduled makespan and the launch status. Arguments: iterations clusters mode
// (mode: sequence | hetero | fake | timeout). In "timeout" the device implementation
// of the first vbd task sleeps 300 ms while the launch's waits are limited to 50 ms:
// the Hetero launch must end with LaunchWaitTimeout instead of waiting.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "ats_launcher.hpp"

struct Run {
    unsigned func, iter, cluster, device;
};

int main(int argc, char** argv) {
    const unsigned constraint_iter_count = argc > 1 ? (unsigned)std::atoi(argv[1]) : 3;
    const unsigned num_clusters = argc > 2 ? (unsigned)std::atoi(argv[2]) : 4;
    const char* mode_name = argc > 3 ? argv[3] : "sequence";
    std::vector<Run> runs;
    std::mutex mu;
    const bool slow = !std::strcmp(mode_name, "timeout");
    bool slept = false;
    auto fn_dispatch = [&](unsigned device, const Launcher::LaunchParam& param) {
        if (slow && device == 1 && param.function_id == Launcher::id_vbd_all_in_one && !slept) {
            slept = true;  // only the device thread reaches this
            std::this_thread::sleep_for(std::chrono::milliseconds(300));
        }
        std::lock_guard<std::mutex> lock(mu);
        runs.push_back({(unsigned)param.function_id, param.iter_idx, param.cluster_idx, device});
    };

    Launcher::Scheduler scheduler;
    {
        Launcher::Implementation ipm_xpbd_cpu(Launcher::DeviceTypeCpu,
                                              [&](const Launcher::LaunchParam& param) { fn_dispatch(0, param); });
        Launcher::Implementation imp_xpbd_gpu(Launcher::DeviceTypeGpu,
                                              [&](const Launcher::LaunchParam& param) { fn_dispatch(1, param); });
        std::vector<Launcher::Implementation> implementation_list_xpbd_cpu_and_gpu = {ipm_xpbd_cpu, imp_xpbd_gpu};

        uint32_t tid_xpbd_predict_position = scheduler.add_task(
            Launcher::Task(Launcher::id_xpbd_predict_position, 0, implementation_list_xpbd_cpu_and_gpu));

        std::vector<uint32_t> constraint_task_orders;
        std::vector<std::vector<uint32_t>> constraint_tasks;
        for (uint32_t iter = 0; iter < constraint_iter_count; iter++) {
            std::vector<uint32_t> curr_tasks;
            for (uint32_t cluster = 0; cluster < num_clusters; cluster++) {
                // the resource list names the cluster's vertex set
                uint32_t tid = scheduler.add_task(Launcher::Task(Launcher::id_vbd_all_in_one, iter, -1u, cluster,
                                                                 std::vector<uint32_t>{cluster},
                                                                 implementation_list_xpbd_cpu_and_gpu));
                scheduler.set_connect(tid_xpbd_predict_position, tid);
                curr_tasks.push_back(tid);
            }
            constraint_tasks.push_back(curr_tasks);
            constraint_task_orders.insert(constraint_task_orders.end(), curr_tasks.begin(), curr_tasks.end());
            if (iter >= 1) {
                const auto& prev_tasks = constraint_tasks[iter - 1];
                for (uint32_t cluster = 0; cluster < prev_tasks.size(); cluster++)
                    scheduler.set_connect(prev_tasks[cluster], curr_tasks[cluster]);
            }
        }
        scheduler.set_constraint_task_orders(constraint_task_orders);
        uint32_t last_node = scheduler.add_task(
            Launcher::Task(Launcher::id_xpbd_constraint_last_node, 0, implementation_list_xpbd_cpu_and_gpu));
        uint32_t tid_xpbd_update_velocity = scheduler.add_task(
            Launcher::Task(Launcher::id_xpbd_update_velocity, 0, implementation_list_xpbd_cpu_and_gpu));
        for (uint32_t left : constraint_tasks.back()) scheduler.set_connect(left, last_node);
        scheduler.set_connect(last_node, tid_xpbd_update_velocity);
    }
    {
        std::vector<std::pair<Launcher::FunctionID, uint32_t>> list_task_id = {
            {Launcher::id_xpbd_predict_position, 0},  {Launcher::id_xpbd_update_velocity, 0},
            {Launcher::id_xpbd_copy_to_cpu_gpu, 0},   {Launcher::id_xpbd_constraint_last_node, 0},
            {Launcher::id_vbd_all_in_one, 0},
        };
        std::vector<std::vector<double>> list_cost;
        std::vector<double> cost_total;
        for (uint32_t cluster = 0; cluster < num_clusters; cluster++)
            list_task_id.push_back({Launcher::id_vbd_all_in_one, cluster});
        for (uint32_t i = 0; i < list_task_id.size(); i++) list_cost.push_back({0.1f, 0.1f});
        scheduler.profile_from(list_task_id, list_cost, cost_total);
    }
    {
        scheduler.communication_cost_matrix_uma = {
            {0.0f, 0.1f},
            {0.1f, 0.0f},
        };
        scheduler.communication_speed_matrix = {};
        scheduler.communication_startup = {0, 0};
    }
    if (scheduler.topological_sort()) {
        scheduler.standardizing_dag();
        scheduler.scheduler_dag();
        scheduler.print_schedule_to_graph_xpbd();
        scheduler.print_speedups_to_each_device();
        scheduler.make_wait_events();
    } else {
        return 3;
    }

    auto fn_task_to_param = [](const Launcher::Task& task) {
        return Launcher::LaunchParam{
            .function_id = task.func_id,
            .iter_idx = task.iter_idx,
            .cluster_idx = task.cluster_idx,
            .is_allocated_to_main_device = task.is_allocated_to_main_device,
            .buffer_idx = task.buffer_idx,
            .left_buffer_idx = task.buffer_left,
            .right_buffer_idx = task.buffer_right,
            .input_buffer_idxs = task.buffer_ins,
        };
    };
    auto mode = Launcher::Scheduler::LaunchModeSequeceHetero;
    if (!std::strcmp(mode_name, "hetero") || slow) mode = Launcher::Scheduler::LaunchModeHetero;
    if (slow) scheduler.set_wait_timeout_ms(50.0);
    if (!std::strcmp(mode_name, "fake")) mode = Launcher::Scheduler::LaunchModeFakeHetero;
    scheduler.set_device_sync(Launcher::DeviceTypeGpu, [] {});  // host-only devices: nothing to drain
    scheduler.launch(mode, fn_task_to_param, false);

    std::printf("{\"status\": %d, \"makespan\": %g, \"tasks\": %zu, \"runs\": [", (int)scheduler.get_last_launch_status(),
                (double)scheduler.get_scheduled_end_time(), scheduler.get_list_task().size());
    for (size_t i = 0; i < runs.size(); ++i)
        std::printf("%s[%u, %d, %u, %u]", i ? ", " : "", runs[i].func, (int)runs[i].iter, runs[i].cluster,
                    runs[i].device);
    std::printf("], \"ids\": {\"predict\": %u, \"vbd\": %u, \"last\": %u, \"update\": %u, \"root\": %u}}\n",
                (unsigned)Launcher::id_xpbd_predict_position, (unsigned)Launcher::id_vbd_all_in_one,
                (unsigned)Launcher::id_xpbd_constraint_last_node, (unsigned)Launcher::id_xpbd_update_velocity,
                (unsigned)Launcher::id_additional_root);
    return 0;
}
