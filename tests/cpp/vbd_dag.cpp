// The VBD task graph of examples/example2_async_iter.cpp:1305-1384 (predict -> one
// id_vbd_all_in_one task per (iteration, colour), colours chained across iterations
// -> last node -> update velocity) with a CUDA implementation registered through
// Launcher::Implementation(DeviceTypeGpu, ...). Runs `frames` frames through the
// scheduler in the requested mode and the same frames through ats_frame on a second
// handle, and prints the largest position difference as JSON (0 = bit-identical).
//
// usage: vbd_dag <grid n> <iterations> <frames> <mode: gpu | hetero | fake | profiled>
// (profiled: costs measured with Scheduler::profile_costs, then the Hetero launch)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ats_cloth.h"
#include "ats_launcher.hpp"

static void check(int r, const char* what) {
    if (r != ATS_OK) {
        std::fprintf(stderr, "%s failed: %s\n", what, ats_last_error());
        std::exit(1);
    }
}

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    const int n = std::atoi(argv[1]), iters = std::atoi(argv[2]), frames = std::atoi(argv[3]);
    const char* mode = argv[4];
    const int nv = n * n, nf = 2 * (n - 1) * (n - 1);
    std::vector<float> pos(3 * nv), mass(nv);
    std::vector<int> faces(3 * nf);
    std::vector<unsigned char> fixed(nv, 0);
    check(ats_grid_mesh(n, ATS_GRID_UNIFORM, pos.data(), faces.data()), "grid");
    check(ats_mass_area_weighted(pos.data(), nv, faces.data(), nf, 0.1f, mass.data()), "mass");
    fixed[0] = fixed[n - 1] = 1;
    ats_instance_desc d{nv, pos.data(), nf, faces.data(), mass.data(), fixed.data(), 1e3f, 1e-2f};
    ats_solver_params prm{1.f / 60.f, 1, iters, 2.f, {0.f, -9.8f, 0.f}, 0, 0};
    ats_cloth *a = nullptr, *b = nullptr;
    check(ats_cloth_create(&d, 1, &prm, &a), "create");
    check(ats_cloth_create(&d, 1, &prm, &b), "create");
    ats_cloth_info info;
    check(ats_cloth_query(a, &info), "query");
    const unsigned ncol = info.num_vertex_colors;

    // fn_dispatch of the GPU implementation (example2_async_iter.cpp:1241-1302)
    auto gpu_dispatch = [&](const Launcher::LaunchParam& p) {
        switch (p.function_id) {
            case Launcher::id_xpbd_predict_position: check(ats_predict_position(a, nullptr), "predict"); break;
            case Launcher::id_vbd_all_in_one: check(ats_vbd_color_sweep(a, (int)p.cluster_idx, nullptr), "sweep"); break;
            case Launcher::id_xpbd_update_velocity: check(ats_update_velocity(a, nullptr), "update"); break;
            default: break;
        }
    };
    // a host-side implementation of the same tasks: it drives the same device
    // work and waits for it, as example2 registers one function for both devices
    auto cpu_dispatch = [&](const Launcher::LaunchParam& p) {
        gpu_dispatch(p);
        std::vector<float> tmp(3 * nv);
        check(ats_get_positions(a, tmp.data(), nullptr), "sync");
    };
    Launcher::Implementation cpu(Launcher::DeviceTypeCpu, cpu_dispatch), gpu(Launcher::DeviceTypeGpu, gpu_dispatch);
    std::vector<Launcher::Implementation> both = {cpu, gpu};

    Launcher::Scheduler s;
    const unsigned t_predict = s.add_task(Launcher::Task(Launcher::id_xpbd_predict_position, 0, both));
    std::vector<unsigned> order;
    std::vector<std::vector<unsigned>> per_iter;
    for (int it = 0; it < iters; ++it) {
        std::vector<unsigned> cur;
        for (unsigned c = 0; c < ncol; ++c) {
            unsigned t = s.add_task(Launcher::Task(Launcher::id_vbd_all_in_one, (unsigned)it, -1u, c, both));
            s.set_connect(t_predict, t);
            cur.push_back(t);
        }
        if (it > 0)
            for (unsigned c = 0; c < ncol; ++c) s.set_connect(per_iter.back()[c], cur[c]);
        order.insert(order.end(), cur.begin(), cur.end());
        per_iter.push_back(cur);
    }
    s.set_constraint_task_orders(order);
    const unsigned t_last = s.add_task(Launcher::Task(Launcher::id_xpbd_constraint_last_node, 0, both));
    const unsigned t_update = s.add_task(Launcher::Task(Launcher::id_xpbd_update_velocity, 0, both));
    for (unsigned t : per_iter.back()) s.set_connect(t, t_last);
    s.set_connect(t_last, t_update);

    auto to_param = [](const Launcher::Task& t) {
        Launcher::LaunchParam p;
        p.function_id = t.func_id;
        p.iter_idx = t.iter_idx;
        p.cluster_idx = t.cluster_idx;
        p.is_allocated_to_main_device = t.is_allocated_to_main_device;
        return p;
    };
    std::vector<std::pair<Launcher::FunctionID, unsigned>> keys;
    std::vector<std::vector<double>> costs;
    if (!std::strcmp(mode, "profiled")) {
        // measured costs on this B200 (host implementation = device work + wait)
        s.profile_costs(to_param, 5, 2, keys, costs);
        check(ats_set_state(a, pos.data(), nullptr, nullptr), "restore");
        std::printf("{\"profiled\": [");
        for (size_t i = 0; i < keys.size(); ++i)
            std::printf("%s[\"%s\", %u, %.5f, %.5f]", i ? ", " : "", Launcher::taskNames.at(keys[i].first).c_str(),
                        keys[i].second, costs[i][0], costs[i][1]);
        std::printf("]}\n");
    } else {
        // computation matrix: the GPU is ten times faster, as a profiled B200 would be
        keys = {{Launcher::id_xpbd_predict_position, 0},
                {Launcher::id_xpbd_update_velocity, 0},
                {Launcher::id_xpbd_constraint_last_node, 0}};
        for (unsigned c = 0; c < ncol; ++c) keys.push_back({Launcher::id_vbd_all_in_one, c});
        costs.assign(keys.size(), std::vector<double>{1.0, 0.1});
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

    Launcher::Scheduler::LaunchMode m = Launcher::Scheduler::LaunchModeGpu;
    if (!std::strcmp(mode, "hetero") || !std::strcmp(mode, "profiled")) m = Launcher::Scheduler::LaunchModeHetero;
    if (!std::strcmp(mode, "fake")) m = Launcher::Scheduler::LaunchModeFakeHetero;
    const unsigned on_gpu = s.get_proc_schedules().size() > 1 ? (unsigned)s.get_proc_schedules()[1].size() : 0u;
    for (int f = 0; f < frames; ++f) {
        s.launch(m, to_param, false);
        check(ats_frame(b, ATS_SOLVER_VBD, nullptr), "frame");
    }
    std::vector<float> xa(3 * nv), xb(3 * nv), va(3 * nv), vb(3 * nv);
    check(ats_get_state(a, xa.data(), va.data(), nullptr), "state");
    check(ats_get_state(b, xb.data(), vb.data(), nullptr), "state");
    double dmax = 0.0, disp = 0.0;
    for (int i = 0; i < 3 * nv; ++i) {
        dmax = std::fmax(dmax, std::fabs((double)xa[i] - xb[i]));
        disp = std::fmax(disp, std::fabs((double)xa[i] - pos[i]));
    }
    std::printf("{\"max_abs_diff\": %.9g, \"max_displacement\": %.6g, \"tasks\": %zu, \"tasks_on_gpu\": %u, "
                "\"makespan\": %.4f, \"cross_device_waits\": %zu}\n",
                dmax, disp, s.get_list_task().size(), on_gpu, s.get_scheduled_end_time(), s.get_wait_events().size());
    ats_cloth_destroy(a);
    ats_cloth_destroy(b);
    return 0;
}
