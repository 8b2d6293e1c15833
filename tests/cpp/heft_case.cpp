// HEFT known-answer driver: reads a DAG and a computation matrix from stdin, runs
// the Launcher scheduler the way examples/example1_heft2002.cpp does (tasks with
// one implementation per processor, speed matrix, no UMA delays, zero start-up),
// and prints the schedule as JSON.
//
// stdin: nprocs ntasks nedges, then ntasks rows of nprocs costs, then nedges lines
// "a b weight" with 1-based task numbers.
#include <cstdio>
#include <vector>

#include "ats_launcher.hpp"

int main() {
    unsigned nprocs = 0, ntasks = 0, nedges = 0;
    if (std::scanf("%u %u %u", &nprocs, &ntasks, &nedges) != 3) return 2;
    Launcher::Scheduler s;
    std::vector<Launcher::Implementation> imps;
    for (unsigned p = 0; p < nprocs; ++p) imps.push_back(Launcher::Implementation(p, [](const Launcher::LaunchParam&) {}));
    std::vector<unsigned> tid(ntasks);
    for (unsigned t = 0; t < ntasks; ++t) tid[t] = s.add_task(Launcher::Task(Launcher::id_task_heft_2002, t + 1, imps));
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
    s.communication_speed_matrix.assign(nprocs, std::vector<float>(nprocs, 1.f));
    for (unsigned p = 0; p < nprocs; ++p) s.communication_speed_matrix[p][p] = 0.f;
    s.communication_cost_matrix_uma = {};
    s.communication_startup.assign(nprocs, 0.f);
    s.summary_of_costs_each_device.assign(nprocs, 0.0);
    for (unsigned p = 0; p < nprocs; ++p)
        for (unsigned t = 0; t < ntasks; ++t)
            s.summary_of_costs_each_device[p] += s.computation_matrix[tid[t]][p] + s.fn_get_inner_communication_cost(p);
    if (!s.topological_sort()) return 3;
    s.standardizing_dag();
    s.scheduler_dag();
    // run the schedule once with every mode that needs no device
    unsigned calls = 0;
    auto to_param = [&](const Launcher::Task& t) {
        Launcher::LaunchParam p;
        p.function_id = t.func_id;
        p.cluster_idx = t.cluster_idx;
        ++calls;
        return p;
    };
    s.launch(Launcher::Scheduler::LaunchModeSequeceHetero, to_param, true);
    const auto speed = s.get_scheduled_speedups();
    std::printf("{\"makespan\": %.4f, \"launched\": %u, \"speedups_percent\": [", s.get_scheduled_end_time(), calls);
    for (size_t p = 0; p < speed.size(); ++p) std::printf("%s%.2f", p ? ", " : "", speed[p] * 100.0);
    std::printf("], \"schedule\": [");
    const auto& ts = s.get_task_schedules();
    for (unsigned t = 0; t < ntasks; ++t)
        std::printf("%s[%u, %u, %.3f, %.3f]", t ? ", " : "", t + 1, ts[tid[t]].proc, ts[tid[t]].start, ts[tid[t]].end);
    std::printf("]}\n");
    return 0;
}
