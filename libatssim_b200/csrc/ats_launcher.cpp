// ats_launcher.cpp -- task DAG, HEFT scheduling and launch for the Launcher API.
//
// Scheduling follows the reference scheduler (src/heterogeneous/launcher.cpp):
//   * topological order: depth-first post-order, reversed (launcher.cpp:25-73, 139-191);
//   * standardizing_dag: one zero-cost root and terminal (:1587-1714);
//   * upward rank with the mean computation cost over the processors that implement a
//     task and a constant mean edge cost of  sum(startup) + (1 + sum(startup))
//     (:1716-2364, RankMetricMEAN), re-chained along set_constraint_task_orders;
//   * HEFT earliest-finish-time with insertion into idle slots (:2369-2401, 2521-2563,
//     2742-2947), communication cost = weight / speed, or the UMA constant delay
//     when that matrix is given (:2465-2484).
// Launch runs on Linux: CPU implementations on the calling thread, GPU
// implementations enqueue on their own CUDA streams; a device-sync hook drains the
// GPU where a host task depends on GPU work and at the end of a launch.

#include "../../include/ats_launcher.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <functional>
#include <mutex>
#include <set>
#include <stack>
#include <thread>

namespace Launcher {

const std::unordered_map<FunctionID, std::string> taskNames = {
#define ATS_LAUNCHER_NAME_ENTRY(name) {name, #name},
    ATS_LAUNCHER_FUNCTION_IDS(ATS_LAUNCHER_NAME_ENTRY)
#undef ATS_LAUNCHER_NAME_ENTRY
};

static const char* name_of(FunctionID f) {
    auto it = taskNames.find(f);
    return it == taskNames.end() ? "unknown" : it->second.c_str();
}

bool Task::has_implementation(const DeviceType& t) const {
    for (const auto& imp : list_implementation)
        if (imp.device == t) return true;
    return false;
}

const Implementation& Task::get_implementation(const DeviceType& t, bool& find) const {
    static const Implementation none;
    for (const auto& imp : list_implementation)
        if (imp.device == t) {
            find = true;
            return imp;
        }
    find = false;
    return list_implementation.empty() ? none : list_implementation[0];
}

void Task::print_with_cluster(const uint tid) const {
    if (iter_idx != -1u)
        std::printf("    Task %u in iteration %2u's cluster %u => %s\n", tid, iter_idx, cluster_idx, name_of(func_id));
    else
        std::printf("    Task %u with cluster %u => %s\n", tid, cluster_idx, name_of(func_id));
}

uint Scheduler::add_task(const Task& task) {
    list_task.push_back(task);
    return (uint)list_task.size() - 1;
}

uint Scheduler::find_task_by_func_id(const FunctionID id) const {
    for (uint t = 0; t < list_task.size(); ++t)
        if (list_task[t].func_id == id) return t;
    return -1u;
}

void Scheduler::set_connect(const uint& a, const uint& b, const float& weight) {
    list_task[a].add_front(b);
    list_task[a].list_weight.push_back(weight);
    list_task[b].add_back(a);
}

float Scheduler::delete_connect(const uint& a, const uint& b) {
    Task& ta = list_task[a];
    Task& tb = list_task[b];
    auto it = std::find(ta.successors.begin(), ta.successors.end(), b);
    if (it == ta.successors.end()) {
        std::fprintf(stderr, "delete_connect: %u is not a successor of %u\n", b, a);
        return 0.f;
    }
    const size_t k = it - ta.successors.begin();
    const float w = ta.list_weight[k];
    ta.successors.erase(it);
    ta.list_weight.erase(ta.list_weight.begin() + k);
    auto jt = std::find(tb.predecessors.begin(), tb.predecessors.end(), a);
    if (jt != tb.predecessors.end()) tb.predecessors.erase(jt);
    return w;
}

bool Scheduler::topological_sort() {
    const uint n = (uint)list_task.size();
    std::vector<uint8_t> state(n, 0);  // 0 new, 1 on the current path, 2 finished
    std::vector<uint> post;
    post.reserve(n);
    bool cyclic = false;
    // iterative DFS: (node, next successor position)
    for (uint s = 0; s < n && !cyclic; ++s) {
        if (state[s]) continue;
        std::stack<std::pair<uint, size_t>> st;
        st.push({s, 0});
        state[s] = 1;
        while (!st.empty() && !cyclic) {
            auto& top = st.top();
            const Task& t = list_task[top.first];
            if (top.second < t.successors.size()) {
                const uint nx = t.successors[top.second++];
                if (state[nx] == 0) {
                    state[nx] = 1;
                    st.push({nx, 0});
                } else if (state[nx] == 1) {
                    cyclic = true;
                }
            } else {
                state[top.first] = 2;
                post.push_back(top.first);
                st.pop();
            }
        }
    }
    if (cyclic) {
        std::fprintf(stderr, "topological_sort: the task graph contains a cycle\n");
        list_order.clear();
        return false;
    }
    list_order.assign(post.rbegin(), post.rend());
    return true;
}

void Scheduler::profile_from(const std::vector<std::pair<FunctionID, uint>>& map_tasks,
                             const std::vector<std::vector<double>>& map_costs, std::vector<double>& cost_total) {
    if (map_costs.empty()) return;
    const uint nprocs = (uint)map_costs.back().size();
    std::vector<double> sum(nprocs, 0.0);
    computation_matrix.assign(list_task.size(), std::vector<float>(nprocs, inf));
    for (uint t = 0; t < list_task.size(); ++t) {
        const Task& task = list_task[t];
        const std::vector<double>* costs = nullptr;
        for (size_t i = 0; i < map_tasks.size(); ++i)
            if (map_tasks[i].first == task.func_id && map_tasks[i].second == task.cluster_idx) {
                costs = &map_costs[i];
                break;
            }
        static const std::vector<double> zeros(16, 0.0);
        if (!costs) {
            std::fprintf(stderr, "profile_from: no cost for task %s / %u\n", name_of(task.func_id), task.cluster_idx);
            costs = &zeros;
        }
        for (uint p = 0; p < nprocs; ++p) {
            const double c = p < costs->size() ? (*costs)[p] : 0.0;
            if (c < 0) {
                std::fprintf(stderr, "profile_from: negative cost for %s\n", name_of(task.func_id));
                return;
            }
            computation_matrix[t][p] = task.has_implementation(p) ? (float)c : inf;
            sum[p] += c;
        }
    }
    if (cost_total.empty()) cost_total = sum;
    summary_of_costs_each_device = cost_total;
}

void Scheduler::profile_costs(const std::function<LaunchParam(const Task&)>& task_to_param, int repeats, uint nprocs,
                              std::vector<std::pair<FunctionID, uint>>& keys, std::vector<std::vector<double>>& costs) {
    keys.clear();
    costs.clear();
    repeats = std::max(1, repeats);
    std::map<std::pair<uint, uint>, uint> seen;  // (func, cluster) -> representative task
    for (uint t = 0; t < list_task.size(); ++t) {
        const auto key = std::make_pair((uint)list_task[t].func_id, list_task[t].cluster_idx);
        if (!seen.count(key)) seen[key] = t;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    for (const auto& kv : seen) {
        const Task& task = list_task[kv.second];
        std::vector<double> row(nprocs, (double)inf);
        for (uint p = 0; p < nprocs; ++p) {
            bool found = false;
            const Implementation& imp = task.get_implementation(p, found);
            if (!found) continue;
            drain(p);
            imp.launch_task(task_to_param(task));  // warm-up
            drain(p);
            auto sit = device_stream.find(p);
            if (p != DeviceTypeCpu && sit != device_stream.end()) {
                // device time between two events on the device's stream
                cudaStream_t st = (cudaStream_t)sit->second;
                if (!e0 && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) {
                    std::fprintf(stderr, "profile_costs: cudaEventCreate failed\n");
                    return;
                }
                cudaEventRecord(e0, st);
                for (int r = 0; r < repeats; ++r) imp.launch_task(task_to_param(task));
                cudaEventRecord(e1, st);
                float ms = 0.f;
                if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                    std::fprintf(stderr, "profile_costs: event timing failed\n");
                    continue;
                }
                row[p] = (double)ms / repeats;
            } else {
                const auto t0 = std::chrono::steady_clock::now();
                for (int r = 0; r < repeats; ++r) imp.launch_task(task_to_param(task));
                drain(p);
                const auto t1 = std::chrono::steady_clock::now();
                row[p] = std::chrono::duration<double, std::milli>(t1 - t0).count() / repeats;
            }
        }
        keys.push_back({task.func_id, task.cluster_idx});
        costs.push_back(row);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
}

void Scheduler::standardizing_dag(const std::vector<std::function<void(const LaunchParam&)>>& empty_fns) {
    const uint nprocs = (uint)communication_startup.size();
    std::vector<Implementation> empty;
    for (uint p = 0; p < nprocs; ++p)
        empty.push_back(Implementation(p, p < empty_fns.size() ? empty_fns[p] : [](const LaunchParam&) {}));
    std::vector<uint> sources;
    for (uint t = 0; t < list_task.size(); ++t)
        if (list_task[t].predecessors.empty()) sources.push_back(t);
    root_node = add_task(Task(id_additional_root, 0, false, true, empty));
    list_task[root_node].is_computation_time_constant = true;
    list_task[root_node].is_empty_node = true;
    computation_matrix.push_back(std::vector<float>(nprocs, 0.f));
    list_order.insert(list_order.begin(), root_node);
    for (uint t : sources) set_connect(root_node, t, 0.f);
    std::vector<uint> sinks;
    for (uint t = 0; t < list_task.size(); ++t)
        if (list_task[t].successors.empty()) sinks.push_back(t);
    terminal_node = add_task(Task(id_additional_terminal, 0, false, true, empty));
    list_task[terminal_node].is_computation_time_constant = true;
    list_task[terminal_node].is_empty_node = true;
    computation_matrix.push_back(std::vector<float>(nprocs, 0.f));
    list_order.push_back(terminal_node);
    for (uint t : sinks) set_connect(t, terminal_node, 0.f);
}

double Scheduler::avg_cost(uint tid, uint nprocs) const {
    double s = 0.0, n = 0.0;
    for (uint p = 0; p < nprocs; ++p)
        if (computation_matrix[tid][p] != inf) {
            s += computation_matrix[tid][p];
            n += 1.0;
        }
    return n > 0 ? s / n : 0.0;
}

void Scheduler::compute_ranku(uint nprocs) {
    const uint n = (uint)list_task.size();
    double startup = 0.0;
    for (uint p = 0; p < nprocs && p < communication_startup.size(); ++p) startup += communication_startup[p];
    const double mean_edge = startup + (1.0 + startup);
    avg_weight.assign(n, {});
    for (uint t = 0; t < n; ++t) avg_weight[t].assign(list_task[t].successors.size(), mean_edge);
    ranku.assign(n, 0.0);
    auto rank_from_successors = [&](uint node) {
        double best = -1.0;
        const Task& t = list_task[node];
        for (size_t j = 0; j < t.successors.size(); ++j) best = std::max(best, avg_weight[node][j] + ranku[t.successors[j]]);
        if (best < 0.0) std::fprintf(stderr, "compute_ranku: task %u has no successor rank\n", node);
        return avg_cost(node, nprocs) + best;
    };
    ranku[terminal_node] = avg_cost(terminal_node, nprocs);
    for (uint i = 1; i < n; ++i) {
        const uint node = list_order[n - 1 - i];
        ranku[node] = rank_from_successors(node);
    }
    ranku[root_node] = inf;
    if (!constraint_task_orders.empty()) {
        // chain the constraint tasks so that their ranks follow the given order
        std::vector<uint8_t> fixed(n, 0);
        const size_t k = constraint_task_orders.size();
        fixed[constraint_task_orders.back()] = 1;
        for (size_t i = 1; i < k; ++i) {
            const uint cur = constraint_task_orders[k - 1 - i], nxt = constraint_task_orders[k - i];
            const double w = avg_weight[cur].empty() ? mean_edge : avg_weight[cur][0];
            ranku[cur] = avg_cost(cur, nprocs) + w + ranku[nxt];
            fixed[cur] = 1;
        }
        for (uint i = 1; i < n; ++i) {
            const uint node = list_order[n - 1 - i];
            if (!fixed[node]) ranku[node] = rank_from_successors(node);
        }
        ranku[root_node] = inf;
    }
}

float Scheduler::fn_get_communication_cost(uint proc, uint pred, uint node) const {
    const Task& pt = list_task[pred];
    auto it = std::find(pt.successors.begin(), pt.successors.end(), node);
    if (it == pt.successors.end()) return 0.f;
    const float w = pt.list_weight[it - pt.successors.begin()];
    if (w == 0.f) return 0.f;
    const uint pp = task_schedules[pred].proc;
    if (!communication_cost_matrix_uma.empty()) return communication_cost_matrix_uma[pp][proc];
    if (pp == proc) return communication_speed_matrix[pp][proc];
    return w / communication_speed_matrix[pp][proc];
}

float Scheduler::fn_get_inner_communication_cost(uint proc) const {
    return !communication_cost_matrix_uma.empty() ? communication_cost_matrix_uma[proc][proc]
                                                  : communication_speed_matrix[proc][proc];
}

ScheduleEvent Scheduler::compute_eft(uint node, uint proc) const {
    float ready = 0.f;
    for (uint pred : list_task[node].predecessors)
        ready = std::max(ready, task_schedules[pred].end + fn_get_communication_cost(proc, pred, node));
    const float ct = computation_matrix[node][proc];
    const float inner = fn_get_inner_communication_cost(proc);
    const auto& jobs = proc_schedules[proc];
    for (size_t i = 0; i < jobs.size(); ++i) {
        const ScheduleEvent& prev = jobs[i];
        if (i == 0 && prev.start > ready + ct + inner) return ScheduleEvent(node, proc, ready, ready + ct);
        const float start = std::max(ready, prev.end + inner);
        if (i + 1 == jobs.size()) return ScheduleEvent(node, proc, start, start + ct);
        if (jobs[i + 1].start - start > ct) return ScheduleEvent(node, proc, start, start + ct);
    }
    return ScheduleEvent(node, proc, ready, ready + ct);
}

void Scheduler::scheduler_dag() {
    const uint nprocs = (uint)communication_startup.size();
    const uint n = (uint)list_task.size();
    if (list_order.size() != n || root_node == -1u || terminal_node == -1u || computation_matrix.size() != n) {
        std::fprintf(stderr, "scheduler_dag: call topological_sort, set the computation matrix and standardizing_dag first\n");
        return;
    }
    compute_ranku(nprocs);
    sorted_nodes.resize(n);
    for (uint t = 0; t < n; ++t) sorted_nodes[t] = t;
    std::stable_sort(sorted_nodes.begin(), sorted_nodes.end(), [&](uint a, uint b) { return ranku[a] > ranku[b]; });
    if (safety_check) {
        std::vector<uint> pos(n);
        for (uint i = 0; i < n; ++i) pos[sorted_nodes[i]] = i;
        for (uint i = 0; i < n; ++i)
            for (uint pred : list_task[sorted_nodes[i]].predecessors)
                if (pos[pred] >= i)
                    std::fprintf(stderr, "scheduler_dag: task %u is ranked before its predecessor %u\n", sorted_nodes[i],
                                 pred);
    }
    if (sorted_nodes[0] != root_node) {
        auto it = std::find(sorted_nodes.begin(), sorted_nodes.end(), root_node);
        std::swap(sorted_nodes[0], *it);
    }
    task_schedules.assign(n, ScheduleEvent());
    proc_schedules.assign(nprocs, {});
    for (uint node : sorted_nodes) {
        ScheduleEvent best(node, 0, inf, inf);
        for (uint p = 0; p < nprocs; ++p) {
            ScheduleEvent e = compute_eft(node, p);
            if (print_detail)
                std::printf("  task %u on proc %u: [%g, %g]\n", node, p, (double)e.start, (double)e.end);
            if (e.start >= inf) {
                std::fprintf(stderr, "scheduler_dag: infinite start for task %u\n", node);
                return;
            }
            if (e.end < best.end) best = e;
        }
        task_schedules[node] = best;
        list_task[node].is_allocated_to_main_device = best.proc == 0;
        auto& jobs = proc_schedules[best.proc];
        jobs.push_back(best);
        std::sort(jobs.begin(), jobs.end());
    }
}

void Scheduler::make_wait_events() {
    wait_events.clear();
    launch_events.clear();
    if (proc_schedules.empty()) return;
    const uint n = (uint)list_task.size();
    for (uint t = 0; t < n; ++t)
        for (uint pred : list_task[t].predecessors)
            if (task_schedules[pred].proc != task_schedules[t].proc)
                wait_events.push_back(WaitEvent{t, task_schedules[t].proc, pred});
    // launch events: split every processor's job list before a task that waits for
    // another processor and after a task that another processor waits for
    launch_events.assign(proc_schedules.size(), {});
    for (uint p = 0; p < proc_schedules.size(); ++p) {
        const auto& jobs = proc_schedules[p];
        LaunchEvent cur;
        bool open = false;
        for (uint i = 0; i < jobs.size(); ++i) {
            const Task& t = list_task[jobs[i].task_id];
            std::vector<uint> waits;
            for (uint pred : t.predecessors)
                if (task_schedules[pred].proc != p) waits.push_back(pred);
            bool signal = false;
            for (uint succ : t.successors) signal |= task_schedules[succ].proc != p;
            if (open && !waits.empty()) {
                launch_events[p].push_back(cur);
                open = false;
            }
            if (!open) {
                cur = LaunchEvent();
                cur.proc = p;
                cur.start_idx = i;
                open = true;
            }
            cur.end_idx = i;
            cur.waits.insert(cur.waits.end(), waits.begin(), waits.end());
            if (signal) {
                cur.signal = true;
                launch_events[p].push_back(cur);
                open = false;
            }
        }
        if (open) launch_events[p].push_back(cur);
    }
}

float Scheduler::get_scheduled_end_time() const {
    float end = 0.f;
    for (const auto& jobs : proc_schedules)
        if (!jobs.empty()) end = std::max(end, jobs.back().end);
    return end;
}

std::vector<float> Scheduler::get_scheduled_speedups() const {
    const float end = get_scheduled_end_time();
    std::vector<float> s(proc_schedules.size(), 0.f);
    for (size_t p = 0; p < s.size() && p < summary_of_costs_each_device.size(); ++p)
        s[p] = (float)((summary_of_costs_each_device[p] - end) / end);
    return s;
}

void Scheduler::print_proc_schedules() const {
    for (size_t p = 0; p < proc_schedules.size(); ++p) {
        std::printf("Processor %zu:\n", p);
        for (const auto& e : proc_schedules[p])
            std::printf("  task %u [%s, cluster %u] from %g to %g\n", e.task_id, name_of(list_task[e.task_id].func_id),
                        list_task[e.task_id].cluster_idx, (double)e.start, (double)e.end);
    }
}

void Scheduler::print_speedups_to_each_device() const {
    const float end = get_scheduled_end_time();
    const auto s = get_scheduled_speedups();
    for (size_t p = 0; p < s.size(); ++p)
        std::printf("Speedup to proc %zu = %4.2f%% (From %4.2f to %4.2f )\n", p, (double)s[p] * 100.0,
                    p < summary_of_costs_each_device.size() ? summary_of_costs_each_device[p] : 0.0, (double)end);
}

void Scheduler::print_sort_by_typology() const {
    for (uint t : list_order)
        std::printf("  task %u in iteration %d cluster %u => %s\n", t, (int)list_task[t].iter_idx, list_task[t].cluster_idx,
                    name_of(list_task[t].func_id));
}

void Scheduler::print_schedule_to_graph_xpbd() const {
    if (proc_schedules.empty()) {
        std::fprintf(stderr, "print_schedule_to_graph_xpbd: no schedule; call scheduler_dag first\n");
        return;
    }
    // colour key: the rank of the task's function id among the scheduled ones, plus
    // its cluster (so the colours of one function sit next to each other)
    std::set<uint> funcs;
    for (const auto& jobs : proc_schedules)
        for (const auto& e : jobs) funcs.insert((uint)list_task[e.task_id].func_id);
    std::map<uint, uint> base;
    uint next = 0;
    for (uint f : funcs) {
        base[f] = next;
        uint maxc = 0;
        for (const auto& t : list_task)
            if ((uint)t.func_id == f) maxc = std::max(maxc, t.cluster_idx);
        next += maxc + 1;
    }
    std::printf("\n Task of each processor\n");
    for (size_t p = 0; p < proc_schedules.size(); ++p) {
        const auto& jobs = proc_schedules[p];
        std::printf("    [");
        for (size_t i = 0; i < jobs.size(); ++i) {
            const ScheduleEvent& e = jobs[i];
            const Task& t = list_task[e.task_id];
            std::printf("(%u, %u, %d, %4.3f, %4.3f)%s", base[(uint)t.func_id] + t.cluster_idx, e.task_id,
                        (int)t.buffer_idx, (double)e.start, (double)e.end, i + 1 < jobs.size() ? ", " : "");
        }
        std::printf("],\n");
        for (size_t i = 0; i < jobs.size(); ++i) {
            const ScheduleEvent& e = jobs[i];
            if (e.task_id < computation_matrix.size() && p < computation_matrix[e.task_id].size() &&
                std::fabs((e.end - e.start) - computation_matrix[e.task_id][p]) > 0.001f)
                std::fprintf(stderr, "   task %u: scheduled length %g does not match its cost %g\n", e.task_id,
                             (double)(e.end - e.start), (double)computation_matrix[e.task_id][p]);
        }
    }
    std::printf("    [");
    for (const WaitEvent& w : wait_events) {
        const ScheduleEvent& in = task_schedules[w.wait_task];
        const ScheduleEvent& cur = task_schedules[w.task_id];
        std::printf("(%u, %u, %u, %u, %4.3f, %4.3f), ", in.proc, w.wait_task, cur.proc, w.task_id, (double)in.end,
                    (double)cur.start);
    }
    std::printf("],\n");
}

void Scheduler::set_device_sync(DeviceType d, std::function<void()> fn) { device_sync[d] = std::move(fn); }

void Scheduler::set_device_stream(DeviceType d, void* cuda_stream) { device_stream[d] = cuda_stream; }

void Scheduler::drain(DeviceType d) const {
    auto it = device_sync.find(d);
    if (it != device_sync.end()) {
        it->second();
        return;
    }
    if (d == DeviceTypeCpu) return;
    auto st = device_stream.find(d);
    const cudaError_t e = st != device_stream.end() ? cudaStreamSynchronize((cudaStream_t)st->second)
                                                    : cudaDeviceSynchronize();
    if (e != cudaSuccess) std::fprintf(stderr, "launch: device drain failed: %s\n", cudaGetErrorString(e));
}

void Scheduler::refit_runtime_cost(const std::vector<float>& runtime_cost_cpu, const std::vector<float>& runtime_cost_gpu) {
    if (launch_events.size() < 2 || proc_schedules.size() < 2) return;
    const std::vector<float>* measured[2] = {&runtime_cost_cpu, &runtime_cost_gpu};
    for (uint p = 0; p < 2; ++p) {
        const auto& events = launch_events[p];
        const auto& jobs = proc_schedules[p];
        const float inner = fn_get_inner_communication_cost(p);
        for (size_t k = 0; k < events.size() && k < measured[p]->size(); ++k) {
            const LaunchEvent& ev = events[k];
            float planned = 0.f;
            uint free_tasks = 0;
            for (uint i = ev.start_idx; i <= ev.end_idx; ++i) {
                const uint tid = jobs[i].task_id;
                planned += computation_matrix[tid][p];
                if (i != ev.end_idx) planned += inner;
                if (!list_task[tid].is_computation_time_constant) ++free_tasks;
            }
            if (free_tasks == 0) continue;
            const float share = ((*measured[p])[k] - planned) / (float)free_tasks;
            for (uint i = ev.start_idx; i <= ev.end_idx; ++i) {
                const uint tid = jobs[i].task_id;
                if (!list_task[tid].is_computation_time_constant)
                    computation_matrix[tid][p] = std::max(computation_matrix[tid][p] + 0.5f * share, 0.f);
            }
        }
    }
}

// LaunchModeHetero: the GPU launch events are issued by a second host thread, the CPU
// ones run on the calling thread, both in schedule order. A GPU event that depends on
// CPU tasks is issued once the CPU thread has finished them (host counter). A CPU
// event that depends on GPU tasks waits until the GPU event holding them is issued,
// then for its completion: the CUDA event recorded after it on the device stream
// (set_device_stream), polled; without a stream, the device drain (the sync hook, or a
// device synchronisation). Every wait is bounded by wait_timeout_ms.
void Scheduler::launch_hetero(const std::function<LaunchParam(const Task&)>& task_to_param, bool fully_not_wait) {
    last_status = LaunchOk;
    if (launch_events.size() < 2 || proc_schedules.size() < 2) {
        std::fprintf(stderr, "launch: Hetero needs scheduler_dag() and make_wait_events() with two processors\n");
        last_status = LaunchMissingImplementation;
        return;
    }
    const auto& cpu_ev = launch_events[0];
    const auto& gpu_ev = launch_events[1];
    const auto& cpu_jobs = proc_schedules[0];
    const auto& gpu_jobs = proc_schedules[1];
    const uint n = (uint)list_task.size();
    std::vector<int> cpu_pos(n, -1), gpu_event_of(n, -1);
    for (uint i = 0; i < cpu_jobs.size(); ++i) cpu_pos[cpu_jobs[i].task_id] = (int)i;
    for (uint g = 0; g < gpu_ev.size(); ++g)
        for (uint i = gpu_ev[g].start_idx; i <= gpu_ev[g].end_idx; ++i) gpu_event_of[gpu_jobs[i].task_id] = (int)g;
    auto sit = device_stream.find(DeviceTypeGpu);
    const bool use_events = sit != device_stream.end();
    cudaStream_t st = use_events ? (cudaStream_t)sit->second : nullptr;
    int device = 0;
    if (use_events) cudaGetDevice(&device);
    const size_t G = gpu_ev.size();
    std::vector<cudaEvent_t> ev_begin(use_events ? G : 0, nullptr), ev_end(use_events ? G : 0, nullptr);
    auto destroy_events = [&] {
        for (auto e : ev_begin)
            if (e) cudaEventDestroy(e);
        for (auto e : ev_end)
            if (e) cudaEventDestroy(e);
    };
    for (size_t g = 0; g < ev_begin.size(); ++g)
        if (cudaEventCreate(&ev_begin[g]) != cudaSuccess || cudaEventCreate(&ev_end[g]) != cudaSuccess) {
            std::fprintf(stderr, "launch: cudaEventCreate failed\n");
            destroy_events();
            last_status = LaunchCudaError;
            return;
        }
    std::mutex mu;
    std::condition_variable cv;
    int cpu_done = 0;       // CPU jobs finished (a prefix of cpu_jobs)
    size_t gpu_issued = 0;  // GPU launch events issued (and their end events recorded)
    std::atomic<int> status{LaunchOk};
    const auto limit = std::chrono::duration<double, std::milli>(wait_timeout_ms);
    std::vector<float> cpu_cost(cpu_ev.size(), 0.f), gpu_cost(G, 0.f);
    auto fail = [&](LaunchStatus s) {
        int ok = LaunchOk;
        status.compare_exchange_strong(ok, (int)s);
        cv.notify_all();
    };
    auto run_task = [&](uint tid, DeviceType d) -> bool {
        const Task& t = list_task[tid];
        bool found = false;
        const Implementation& imp = t.get_implementation(d, found);
        if (!found) {
            std::fprintf(stderr, "launch: task %u (%s) has no implementation for device %u\n", tid, name_of(t.func_id), d);
            fail(LaunchMissingImplementation);
            return false;
        }
        try {
            imp.launch_task(task_to_param(t));
        } catch (...) {
            std::fprintf(stderr, "launch: task %u (%s) threw\n", tid, name_of(t.func_id));
            fail(LaunchTaskFailed);
            return false;
        }
        return true;
    };
    std::thread gpu_thread([&] {
        if (use_events) cudaSetDevice(device);
        for (size_t g = 0; g < G && status.load() == LaunchOk; ++g) {
            const LaunchEvent& e = gpu_ev[g];
            int need = 0;
            for (uint w : e.waits)
                if (cpu_pos[w] >= 0) need = std::max(need, cpu_pos[w] + 1);
            if (!fully_not_wait && need > 0) {
                std::unique_lock<std::mutex> lk(mu);
                if (!cv.wait_for(lk, limit, [&] { return cpu_done >= need || status.load() != LaunchOk; })) {
                    lk.unlock();
                    std::fprintf(stderr, "launch: GPU event %zu waited too long for CPU task %d\n", g, need - 1);
                    fail(LaunchWaitTimeout);
                    break;
                }
                if (status.load() != LaunchOk) break;
            }
            const auto t0 = std::chrono::steady_clock::now();
            if (use_events) cudaEventRecord(ev_begin[g], st);
            bool ok = true;
            for (uint i = e.start_idx; i <= e.end_idx && ok; ++i) ok = run_task(gpu_jobs[i].task_id, DeviceTypeGpu);
            if (use_events) cudaEventRecord(ev_end[g], st);
            else gpu_cost[g] = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            {
                std::lock_guard<std::mutex> lk(mu);
                gpu_issued = g + 1;
            }
            cv.notify_all();
            if (!ok) break;
        }
    });
    // waits until GPU launch event g is issued, then until it has completed
    auto wait_gpu_event = [&](size_t g) -> bool {
        {
            std::unique_lock<std::mutex> lk(mu);
            if (!cv.wait_for(lk, limit, [&] { return gpu_issued > g || status.load() != LaunchOk; })) {
                lk.unlock();
                std::fprintf(stderr, "launch: GPU event %zu was not issued in time\n", g);
                fail(LaunchWaitTimeout);
                return false;
            }
            if (gpu_issued <= g) return false;
        }
        if (!use_events) {
            drain(DeviceTypeGpu);
            return true;
        }
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t q = cudaEventQuery(ev_end[g]);
            if (q == cudaSuccess) return true;
            if (q != cudaErrorNotReady) {
                std::fprintf(stderr, "launch: GPU event %zu: %s\n", g, cudaGetErrorString(q));
                fail(LaunchCudaError);
                return false;
            }
            if (std::chrono::steady_clock::now() - t0 > limit) {
                std::fprintf(stderr, "launch: GPU event %zu did not complete in time\n", g);
                fail(LaunchWaitTimeout);
                return false;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    };
    for (size_t c = 0; c < cpu_ev.size() && status.load() == LaunchOk; ++c) {
        const LaunchEvent& e = cpu_ev[c];
        bool ok = true;
        if (!fully_not_wait) {
            int last = -1;
            for (uint w : e.waits) last = std::max(last, gpu_event_of[w]);
            if (last >= 0) ok = wait_gpu_event((size_t)last);  // one stream: earlier events complete first
        }
        if (!ok) break;
        const auto t0 = std::chrono::steady_clock::now();
        for (uint i = e.start_idx; i <= e.end_idx && ok; ++i) ok = run_task(cpu_jobs[i].task_id, DeviceTypeCpu);
        cpu_cost[c] = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        {
            std::lock_guard<std::mutex> lk(mu);
            cpu_done = (int)e.end_idx + 1;
        }
        cv.notify_all();
        if (!ok) break;
    }
    gpu_thread.join();
    if (status.load() == LaunchOk && G > 0 && !fully_not_wait) {
        if (use_events) wait_gpu_event(G - 1);
        else drain(DeviceTypeGpu);
    }
    if (status.load() == LaunchOk) {
        for (size_t g = 0; g < ev_begin.size(); ++g) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ev_begin[g], ev_end[g]) == cudaSuccess) gpu_cost[g] = ms;
        }
        last_runtime_costs = {cpu_cost, gpu_cost};
        if (runtime_refit && !fully_not_wait) refit_runtime_cost(cpu_cost, gpu_cost);
    } else if (use_events) {
        cudaStreamSynchronize(st);  // nothing of this launch stays in flight
    }
    destroy_events();
    last_status = (LaunchStatus)status.load();
}

void Scheduler::launch(LaunchMode mode, const std::function<LaunchParam(const Task&)>& task_to_param, bool fully_not_wait,
                       const std::vector<std::function<void()>>& /*assemble_impl*/) {
    last_status = LaunchOk;
    const std::vector<uint>& order = !sorted_nodes.empty() ? sorted_nodes : list_order;
    if (order.empty()) {
        std::fprintf(stderr, "launch: neither a topological nor a ranked order; call topological_sort first\n");
        return;
    }
    auto run = [&](uint tid, DeviceType d, bool& found) {
        const Task& t = list_task[tid];
        const Implementation& imp = t.get_implementation(d, found);
        if (!found && d != DeviceTypeCpu) drain(d);
        imp.launch_task(task_to_param(t));
    };
    if (mode == LaunchModeCpu) {
        for (uint tid : order) {
            bool found;
            if (!list_task[tid].has_implementation(DeviceTypeCpu)) {
                std::fprintf(stderr, "launch: task %u has no CPU implementation\n", tid);
                return;
            }
            run(tid, DeviceTypeCpu, found);
        }
        return;
    }
    if (mode == LaunchModeGpu) {
        for (uint tid : order) {
            bool found;
            run(tid, DeviceTypeGpu, found);
        }
        if (!fully_not_wait) drain(DeviceTypeGpu);
        return;
    }
    if (proc_schedules.empty()) {
        std::fprintf(stderr, "launch: this mode needs scheduler_dag() first\n");
        return;
    }
    // scheduled modes: tasks in order of scheduled start; ties (a zero-length task and
    // its successor start together) go by end time, then by topological position, so a
    // task never runs before a predecessor that the schedule placed at the same instant
    std::vector<uint> topo_pos(list_task.size(), 0);
    for (size_t i = 0; i < order.size(); ++i)
        if (order[i] < topo_pos.size()) topo_pos[order[i]] = (uint)i;
    std::vector<ScheduleEvent> plan;
    for (const auto& jobs : proc_schedules) plan.insert(plan.end(), jobs.begin(), jobs.end());
    std::stable_sort(plan.begin(), plan.end(), [&](const ScheduleEvent& a, const ScheduleEvent& b) {
        if (a.start != b.start) return a.start < b.start;
        if (a.end != b.end) return a.end < b.end;
        return topo_pos[a.task_id] < topo_pos[b.task_id];
    });
    if (mode == LaunchModePartialCPU || mode == LaunchModePartialGPU) {
        const uint want = mode == LaunchModePartialCPU ? 0u : 1u;
        for (const auto& e : plan)
            if (e.proc == want) {
                bool found;
                run(e.task_id, want, found);
            }
        if (!fully_not_wait && want != DeviceTypeCpu) drain(want);
        return;
    }
    if (mode == LaunchModeSequeceHetero) {
        for (const auto& e : plan) {
            bool found;
            run(e.task_id, DeviceTypeCpu, found);
        }
        return;
    }
    if (mode == LaunchModeHetero || mode == LaunchModeProgressiveHetero) {
        launch_hetero(task_to_param, fully_not_wait);
        return;
    }
    // FakeHetero: each task on its scheduled device, one at a time in order of
    // scheduled start, the GPU drained after every task.
    const bool synchronous = mode == LaunchModeFakeHetero;
    std::vector<uint8_t> pending(list_task.size(), 0);  // device task enqueued, not yet drained
    for (const auto& e : plan) {
        const Task& t = list_task[e.task_id];
        if (e.proc == DeviceTypeCpu) {
            bool wait = false;
            for (uint pred : t.predecessors) wait |= pending[pred] != 0;
            if (wait) {
                drain(DeviceTypeGpu);
                std::fill(pending.begin(), pending.end(), 0);
            }
            bool found;
            run(e.task_id, DeviceTypeCpu, found);
        } else {
            bool found;
            run(e.task_id, e.proc, found);
            pending[e.task_id] = 1;
            if (synchronous) {
                drain(e.proc);
                pending[e.task_id] = 0;
            }
        }
    }
    if (!fully_not_wait) drain(DeviceTypeGpu);
}

}  // namespace Launcher
