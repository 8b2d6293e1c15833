// The VBD task graph of examples/example2_async_iter.cpp:1305-1384 through the Launcher
// API with two real implementations per task:
//   GPU  the CUDA solver through the C ABI (ats_predict_position, ats_vbd_color_sweep,
//        ats_update_velocity), enqueued on the legacy default stream;
//   CPU  the CPU oracle's per-step entry points (ato_predict, ato_vbd_color, ato_update)
//        on a host copy of the same cloth.
// Two cloths (grid sides n and n + 8) are advanced together; each has its own chain
// predict -> (iteration, colour) tasks in sweep order -> last node -> update, so each
// cloth's tasks form a total order, whichever device runs them. The positions follow
// the tasks: a task whose cloth was last touched on the other device first copies the
// current iterate across (ats_get_positions / ats_set_positions). The instance of a
// task travels in its resource list (the Task constructor with resources,
// launcher.h:643-645) and reaches the implementations as LaunchParam::buffer_idx.
//
// usage: vbd_dag <n> <iterations> <frames> <mode>
//   gpu | cpu   every task on one device (LaunchModeGpu / LaunchModeCpu)
//   fake        the HEFT schedule, each task on its device, one at a time (FakeHetero)
//   hetero      the same schedule with both devices at once (Hetero: GPU tasks from a
//               second host thread, ordered by CUDA events)
//   profiled    costs measured by Scheduler::profile_costs (CUDA events on the GPU
//               stream, host clock on the CPU), then Hetero
// With fake / hetero the computation matrix makes both devices equally fast, so HEFT
// gives each device work. Prints one JSON line: launch status, tasks per device, an
// FNV-1a digest of the final positions (equal digests = bit-identical runs), and the
// relative L2 distance to the same frames run by the CUDA solver alone (ats_frame) and
// by the oracle alone.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ats_cloth.h"
#include "ats_launcher.hpp"

extern "C" {
// CPU oracle (oracle/ats_oracle.cpp), test infrastructure
struct ato_params {
    float implicit_dt;
    int num_substep;
    int iterations;
    float k_stretch;
    float k_bend;
    float damping;
    float gravity[3];
    int threads;
};
void* ato_scene_create(const float* pos, int nv, const int* faces, int nf, const float* mass, const unsigned char* fixed,
                       const ato_params* prm);
void ato_scene_destroy(void* h);
void ato_set_state(void* h, const float* x, const float* v);
void ato_get_state(void* h, float* x, float* v);
void ato_frame(void* h, int solver, double* energy_log, int with_bending, double* residual_log);
void ato_frame_begin(void* h);
void ato_predict(void* h);
void ato_vbd_color(void* h, int c);
void ato_update(void* h);
void ato_get_x(void* h, float* x);
void ato_set_x(void* h, const float* x);
}

static void check(int r, const char* what) {
    if (r != ATS_OK) {
        std::fprintf(stderr, "%s failed: %s\n", what, ats_last_error());
        std::exit(1);
    }
}

struct Cloth {
    int n = 0, nv = 0, nf = 0;
    std::vector<float> pos, mass;
    std::vector<int> faces;
    std::vector<unsigned char> fixed;
    ats_cloth* gpu = nullptr;    // scheduled run, device side
    void* cpu = nullptr;         // scheduled run, host side
    ats_cloth* alone = nullptr;  // the same frames by ats_frame alone
    void* oracle = nullptr;      // the same frames by the oracle alone
    int owner = 0;               // device holding the current iterate (0 CPU, 1 GPU)
    int updated_on = 1;          // device that ran the last velocity update
    std::vector<float> buf, vbuf;
};

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    const int n = std::atoi(argv[1]), iters = std::atoi(argv[2]), frames = std::atoi(argv[3]);
    const char* mode = argv[4];
    ats_stream st = nullptr;  // the legacy default stream carries every GPU task
    const ats_solver_params prm{1.f / 60.f, 1, iters, 2.f, {0.f, -9.8f, 0.f}, 0, 0};
    const ato_params oprm{1.f / 60.f, 1, iters, 1e3f, 1e-2f, 2.f, {0.f, -9.8f, 0.f}, 2};
    Cloth cl[2];
    for (int k = 0; k < 2; ++k) {
        Cloth& c = cl[k];
        c.n = n + 8 * k;
        c.nv = c.n * c.n;
        c.nf = 2 * (c.n - 1) * (c.n - 1);
        c.pos.resize(3 * c.nv);
        c.faces.resize(3 * c.nf);
        c.mass.resize(c.nv);
        c.fixed.assign(c.nv, 0);
        check(ats_grid_mesh(c.n, ATS_GRID_UNIFORM, c.pos.data(), c.faces.data()), "grid");
        check(ats_mass_area_weighted(c.pos.data(), c.nv, c.faces.data(), c.nf, 0.1f, c.mass.data()), "mass");
        c.fixed[0] = c.fixed[c.n - 1] = 1;
        ats_instance_desc d{c.nv, c.pos.data(), c.nf, c.faces.data(), c.mass.data(), c.fixed.data(), 1e3f, 1e-2f};
        check(ats_cloth_create(&d, 1, &prm, &c.gpu), "create");
        check(ats_cloth_create(&d, 1, &prm, &c.alone), "create");
        c.cpu = ato_scene_create(c.pos.data(), c.nv, c.faces.data(), c.nf, c.mass.data(), c.fixed.data(), &oprm);
        c.oracle = ato_scene_create(c.pos.data(), c.nv, c.faces.data(), c.nf, c.mass.data(), c.fixed.data(), &oprm);
        c.buf.resize(3 * c.nv);
        c.vbuf.resize(3 * c.nv);
    }
    ats_cloth_info info;
    check(ats_cloth_query(cl[0].gpu, &info), "query");
    const unsigned ncol = (unsigned)info.num_vertex_colors;

    // the current iterate follows the task to its device
    auto to_gpu = [&](Cloth& c) {
        if (c.owner == 1) return;
        ato_get_x(c.cpu, c.buf.data());
        check(ats_set_positions(c.gpu, c.buf.data(), st), "to gpu");
        c.owner = 1;
    };
    auto to_cpu = [&](Cloth& c) {
        if (c.owner == 0) return;
        check(ats_get_positions(c.gpu, c.buf.data(), st), "to cpu");
        ato_set_x(c.cpu, c.buf.data());
        c.owner = 0;
    };
    auto gpu_dispatch = [&](const Launcher::LaunchParam& p) {
        if (p.buffer_idx > 1) return;  // root / terminal
        Cloth& c = cl[p.buffer_idx];
        switch (p.function_id) {
            case Launcher::id_xpbd_predict_position:
                check(ats_predict_position(c.gpu, st), "predict");
                c.owner = 1;
                break;
            case Launcher::id_vbd_all_in_one:
                to_gpu(c);
                check(ats_vbd_color_sweep(c.gpu, (int)p.cluster_idx, st), "sweep");
                break;
            case Launcher::id_xpbd_update_velocity:
                to_gpu(c);
                check(ats_update_velocity(c.gpu, st), "update");
                c.updated_on = 1;
                break;
            default: break;
        }
    };
    auto cpu_dispatch = [&](const Launcher::LaunchParam& p) {
        if (p.buffer_idx > 1) return;
        Cloth& c = cl[p.buffer_idx];
        switch (p.function_id) {
            case Launcher::id_xpbd_predict_position:
                ato_predict(c.cpu);
                c.owner = 0;
                break;
            case Launcher::id_vbd_all_in_one:
                to_cpu(c);
                ato_vbd_color(c.cpu, (int)p.cluster_idx);
                break;
            case Launcher::id_xpbd_update_velocity:
                to_cpu(c);
                ato_update(c.cpu);
                c.updated_on = 0;
                break;
            default: break;
        }
    };
    Launcher::Implementation cpu(Launcher::DeviceTypeCpu, cpu_dispatch), gpu(Launcher::DeviceTypeGpu, gpu_dispatch);
    const std::vector<Launcher::Implementation> both = {cpu, gpu};

    Launcher::Scheduler s;
    std::vector<unsigned> order;
    for (unsigned k = 0; k < 2; ++k) {
        const std::vector<uint32_t> res = {k};
        unsigned prev = s.add_task(Launcher::Task(Launcher::id_xpbd_predict_position, -1u, -1u, 0, res, both));
        for (int it = 0; it < iters; ++it)
            for (unsigned c = 0; c < ncol; ++c) {
                unsigned t = s.add_task(Launcher::Task(Launcher::id_vbd_all_in_one, (unsigned)it, -1u, c, res, both));
                s.set_connect(prev, t);
                order.push_back(t);
                prev = t;
            }
        const unsigned last = s.add_task(Launcher::Task(Launcher::id_xpbd_constraint_last_node, -1u, -1u, 0, res, both));
        const unsigned upd = s.add_task(Launcher::Task(Launcher::id_xpbd_update_velocity, -1u, -1u, 0, res, both));
        s.set_connect(prev, last);
        s.set_connect(last, upd);
    }
    s.set_constraint_task_orders(order);
    auto to_param = [](const Launcher::Task& t) {
        Launcher::LaunchParam p;
        p.function_id = t.func_id;
        p.iter_idx = t.iter_idx;
        p.cluster_idx = t.cluster_idx;
        p.is_allocated_to_main_device = t.is_allocated_to_main_device;
        p.buffer_idx = t.resources.empty() ? 2u : t.resources[0];
        return p;
    };
    s.set_device_stream(Launcher::DeviceTypeGpu, st);

    std::vector<std::pair<Launcher::FunctionID, unsigned>> keys = {{Launcher::id_xpbd_predict_position, 0},
                                                                   {Launcher::id_xpbd_update_velocity, 0},
                                                                   {Launcher::id_xpbd_constraint_last_node, 0}};
    for (unsigned c = 0; c < ncol; ++c) keys.push_back({Launcher::id_vbd_all_in_one, c});
    std::vector<std::vector<double>> costs(keys.size(), std::vector<double>{1.0, 1.0});
    if (!std::strcmp(mode, "profiled")) {
        for (auto& c : cl) ato_frame_begin(c.cpu);
        s.profile_costs(to_param, 5, 2, keys, costs);
        std::printf("{\"profiled\": [");
        for (size_t i = 0; i < keys.size(); ++i)
            std::printf("%s[\"%s\", %u, %.5f, %.5f]", i ? ", " : "", Launcher::taskNames.at(keys[i].first).c_str(),
                        keys[i].second, costs[i][0], costs[i][1]);
        std::printf("]}\n");
        for (auto& c : cl) {  // back to rest on both sides
            check(ats_set_state(c.gpu, c.pos.data(), nullptr, st), "restore");
            std::vector<float> zero(3 * c.nv, 0.f);
            ato_set_state(c.cpu, c.pos.data(), zero.data());
            c.owner = 1;
            c.updated_on = 1;
        }
    }
    std::vector<double> total;
    s.profile_from(keys, costs, total);
    s.communication_cost_matrix_uma = {{0.0f, 0.1f}, {0.1f, 0.0f}};
    s.communication_speed_matrix = {};
    s.communication_startup = {0.f, 0.f};
    if (!s.topological_sort()) return 3;
    s.standardizing_dag();
    s.scheduler_dag();
    s.make_wait_events();
    unsigned on_dev[2] = {0, 0};
    for (const auto& e : s.get_task_schedules())
        if (s.get_list_task()[e.task_id].func_id == Launcher::id_vbd_all_in_one) ++on_dev[e.proc];

    Launcher::Scheduler::LaunchMode m = Launcher::Scheduler::LaunchModeHetero;
    if (!std::strcmp(mode, "gpu")) m = Launcher::Scheduler::LaunchModeGpu;
    if (!std::strcmp(mode, "cpu")) m = Launcher::Scheduler::LaunchModeCpu;
    if (!std::strcmp(mode, "fake")) m = Launcher::Scheduler::LaunchModeFakeHetero;
    int status = 0;
    for (int f = 0; f < frames; ++f) {
        // both sides start the frame from the state of the side that ended the last one
        for (auto& c : cl) {
            if (c.updated_on == 0) {
                ato_get_state(c.cpu, c.buf.data(), c.vbuf.data());
                check(ats_set_state(c.gpu, c.buf.data(), c.vbuf.data(), st), "sync to gpu");
            } else {
                check(ats_get_state(c.gpu, c.buf.data(), c.vbuf.data(), st), "sync to cpu");
                ato_set_state(c.cpu, c.buf.data(), c.vbuf.data());
            }
            ato_frame_begin(c.cpu);
            c.owner = 1;
        }
        s.launch(m, to_param, false);
        status |= (int)s.get_last_launch_status();
        for (auto& c : cl) {
            check(ats_frame(c.alone, ATS_SOLVER_VBD, nullptr), "frame");
            ato_frame(c.oracle, 0, nullptr, 0, nullptr);
        }
    }
    uint64_t digest = 1469598103934665603ull;
    double d_alone = 0, n_alone = 0, d_oracle = 0, n_oracle = 0, disp = 0;
    for (auto& c : cl) {
        std::vector<float> x(3 * c.nv), v(3 * c.nv), xa(3 * c.nv), xo(3 * c.nv);
        if (c.updated_on == 0) ato_get_state(c.cpu, x.data(), v.data());
        else check(ats_get_state(c.gpu, x.data(), v.data(), st), "state");
        check(ats_get_state(c.alone, xa.data(), v.data(), st), "state");
        ato_get_state(c.oracle, xo.data(), v.data());
        const unsigned char* b = (const unsigned char*)x.data();
        for (size_t i = 0; i < x.size() * sizeof(float); ++i) digest = (digest ^ b[i]) * 1099511628211ull;
        for (size_t i = 0; i < x.size(); ++i) {
            d_alone += ((double)x[i] - xa[i]) * ((double)x[i] - xa[i]);
            n_alone += (double)xa[i] * xa[i];
            d_oracle += ((double)x[i] - xo[i]) * ((double)x[i] - xo[i]);
            n_oracle += (double)xo[i] * xo[i];
            disp = std::fmax(disp, std::fabs((double)x[i] - c.pos[i]));
        }
    }
    const auto& rc = s.get_last_runtime_costs();
    std::printf("{\"status\": %d, \"tasks\": %zu, \"sweeps_on_cpu\": %u, \"sweeps_on_gpu\": %u, \"digest\": \"%016llx\", "
                "\"rel_l2_vs_gpu_alone\": %.3e, \"rel_l2_vs_oracle_alone\": %.3e, \"max_displacement\": %.6g, "
                "\"makespan\": %.4f, \"cross_device_waits\": %zu, \"launch_events\": [%zu, %zu], "
                "\"measured_events\": [%zu, %zu]}\n",
                status, s.get_list_task().size(), on_dev[0], on_dev[1], (unsigned long long)digest,
                std::sqrt(d_alone / n_alone), std::sqrt(d_oracle / n_oracle), disp, s.get_scheduled_end_time(),
                s.get_wait_events().size(), s.get_launch_events()[0].size(), s.get_launch_events()[1].size(),
                rc.empty() ? (size_t)0 : rc[0].size(), rc.empty() ? (size_t)0 : rc[1].size());
    for (auto& c : cl) {
        ats_cloth_destroy(c.gpu);
        ats_cloth_destroy(c.alone);
        ato_scene_destroy(c.cpu);
        ato_scene_destroy(c.oracle);
    }
    return 0;
}
