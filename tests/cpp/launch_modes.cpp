// Launch-mode driver for the Launcher API with two host-only "devices": reads a DAG
// and a two-column computation matrix from stdin (the heft_case format), schedules it
// with HEFT, then runs it in every launch mode. Both implementations of a task only
// record (task number, device) in execution order; the device-1 sync hook records a
// drain as (0, 2). Prints, per mode, the execution log, and the schedule's processor
// per task. The Hetero mode runs device-1 tasks from a second host thread, so the log
// is guarded by a mutex and its order is the order of execution.
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "ats_launcher.hpp"

int main() {
    unsigned nprocs = 0, ntasks = 0, nedges = 0;
    if (std::scanf("%u %u %u", &nprocs, &ntasks, &nedges) != 3 || nprocs != 2) return 2;
    std::vector<std::pair<unsigned, unsigned>> log;
    std::mutex log_mu;
    unsigned drains = 0;
    auto impl = [&](unsigned dev) {
        return Launcher::Implementation(dev, [&log, &log_mu, dev](const Launcher::LaunchParam& p) {
            std::lock_guard<std::mutex> lock(log_mu);
            if (p.iter_idx >= 1) log.push_back({p.iter_idx, dev});
        });
    };
    const std::vector<Launcher::Implementation> both = {impl(0), impl(1)};
    Launcher::Scheduler s;
    std::vector<unsigned> tid(ntasks);
    for (unsigned t = 0; t < ntasks; ++t)
        tid[t] = s.add_task(Launcher::Task(Launcher::id_task_heft_2002, t + 1, -1u, 0, both));
    s.computation_matrix.assign(ntasks, std::vector<float>(nprocs, 0.f));
    for (unsigned t = 0; t < ntasks; ++t)
        for (unsigned p = 0; p < nprocs; ++p)
            if (std::scanf("%f", &s.computation_matrix[tid[t]][p]) != 1) return 2;
    for (unsigned e = 0; e < nedges; ++e) {
        unsigned a, b;
        float w;
        if (std::scanf("%u %u %f", &a, &b, &w) != 3) return 2;
        s.set_connect(tid[a - 1], tid[b - 1], w);
    }
    s.communication_speed_matrix = {{0.f, 1.f}, {1.f, 0.f}};
    s.communication_cost_matrix_uma = {};
    s.communication_startup = {0.f, 0.f};
    s.summary_of_costs_each_device.assign(nprocs, 0.0);
    if (!s.topological_sort()) return 3;
    s.standardizing_dag();
    s.scheduler_dag();
    s.make_wait_events();
    s.set_device_sync(1, [&] {
        std::lock_guard<std::mutex> lock(log_mu);
        ++drains;
        log.push_back({0u, 2u});  // a drain of device 1, in execution order
    });
    auto to_param = [](const Launcher::Task& t) {
        Launcher::LaunchParam p;
        p.function_id = t.func_id;
        p.iter_idx = t.iter_idx == -1u ? 0u : t.iter_idx;
        p.is_allocated_to_main_device = t.is_allocated_to_main_device;
        return p;
    };
    const std::pair<const char*, Launcher::Scheduler::LaunchMode> modes[] = {
        {"cpu", Launcher::Scheduler::LaunchModeCpu},
        {"gpu", Launcher::Scheduler::LaunchModeGpu},
        {"partial_cpu", Launcher::Scheduler::LaunchModePartialCPU},
        {"partial_gpu", Launcher::Scheduler::LaunchModePartialGPU},
        {"sequence_hetero", Launcher::Scheduler::LaunchModeSequeceHetero},
        {"fake_hetero", Launcher::Scheduler::LaunchModeFakeHetero},
        {"hetero", Launcher::Scheduler::LaunchModeHetero},
    };
    std::printf("{\"proc\": [");
    const auto& ts = s.get_task_schedules();
    for (unsigned t = 0; t < ntasks; ++t) std::printf("%s%u", t ? ", " : "", ts[tid[t]].proc);
    std::printf("], \"modes\": {");
    bool first = true;
    for (const auto& m : modes) {
        log.clear();
        drains = 0;
        s.launch(m.second, to_param, false);
        std::printf("%s\"%s\": {\"status\": %d, \"drains\": %u, \"log\": [", first ? "" : ", ", m.first,
                    (int)s.get_last_launch_status(), drains);
        for (size_t i = 0; i < log.size(); ++i) std::printf("%s[%u, %u]", i ? ", " : "", log[i].first, log[i].second);
        std::printf("]}");
        first = false;
    }
    std::printf("}}\n");
    return 0;
}
