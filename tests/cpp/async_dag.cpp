// Two-device asynchronous iteration of examples/example2_async_iter.cpp:1160-1200 driven
// by the Launcher: from a common fork point the CPU and the B200 each iterate their own
// copy of the positions, then the copies are merged by Core::read_and_solve_conflict
// (xpbd_constraints.h:815-869), and the merged positions are the next fork point.
// Per frame:
//   predict (GPU) -> R rounds of [ fork (GPU: ats_async_fork, the CPU copy takes the
//   fork point; id_xpbd_copy_to_cpu_gpu) -> K iterations x colours on each device, each
//   on its own copy (id_vbd_all_in_one; the CPU's by the oracle's per-step functions) ->
//   merge (GPU: ats_async_merge with the CPU copy, weight 0.5;
//   id_xpbd_read_and_solve_conflict) ] -> last node -> update (GPU).
// Every task has an implementation on one device only, so the HEFT schedule puts each
// chain on its device and the two chains of a round overlap in a Hetero launch.
//
// usage: async_dag <n> <rounds> <iterations per round> <frames> <mode: fake | hetero>
// Prints one JSON line: launch status, tasks per device, merges run, an FNV-1a digest
// of the final positions (equal digests = bit-identical runs) and the relative L2
// distance to the same frames solved by plain VBD on the B200 with R x K iterations.
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
void ato_frame_begin(void* h);
void ato_vbd_color(void* h, int c);
void ato_get_x(void* h, float* x);
void ato_set_x(void* h, const float* x);
}

static void check(int r, const char* what) {
    if (r != ATS_OK) {
        std::fprintf(stderr, "%s failed: %s\n", what, ats_last_error());
        std::exit(1);
    }
}

int main(int argc, char** argv) {
    if (argc < 6) return 2;
    const int n = std::atoi(argv[1]), rounds = std::atoi(argv[2]), k_iters = std::atoi(argv[3]);
    const int frames = std::atoi(argv[4]);
    const char* mode = argv[5];
    ats_stream st = nullptr;
    const int nv = n * n, nf = 2 * (n - 1) * (n - 1);
    std::vector<float> pos(3 * nv), mass(nv), buf(3 * nv), vbuf(3 * nv);
    std::vector<int> faces(3 * nf);
    std::vector<unsigned char> fixed(nv, 0);
    check(ats_grid_mesh(n, ATS_GRID_UNIFORM, pos.data(), faces.data()), "grid");
    check(ats_mass_area_weighted(pos.data(), nv, faces.data(), nf, 0.1f, mass.data()), "mass");
    fixed[0] = fixed[n - 1] = 1;
    ats_instance_desc d{nv, pos.data(), nf, faces.data(), mass.data(), fixed.data(), 1e3f, 1e-2f};
    const ats_solver_params prm{1.f / 60.f, 1, rounds * k_iters, 2.f, {0.f, -9.8f, 0.f}, 0, 0};
    const ato_params oprm{1.f / 60.f, 1, rounds * k_iters, 1e3f, 1e-2f, 2.f, {0.f, -9.8f, 0.f}, 2};
    ats_cloth *gpu = nullptr, *alone = nullptr;
    check(ats_cloth_create(&d, 1, &prm, &gpu), "create");
    check(ats_cloth_create(&d, 1, &prm, &alone), "create");
    void* cpu = ato_scene_create(pos.data(), nv, faces.data(), nf, mass.data(), fixed.data(), &oprm);
    ats_cloth_info info;
    check(ats_cloth_query(gpu, &info), "query");
    const unsigned ncol = (unsigned)info.num_vertex_colors;
    int merges = 0;

    auto gpu_dispatch = [&](const Launcher::LaunchParam& p) {
        switch (p.function_id) {
            case Launcher::id_xpbd_predict_position: check(ats_predict_position(gpu, st), "predict"); break;
            case Launcher::id_xpbd_copy_to_cpu_gpu:  // fork: both copies start from the current iterate
                check(ats_async_fork(gpu, st), "fork");
                check(ats_get_positions(gpu, buf.data(), st), "fork copy");
                ato_set_x(cpu, buf.data());
                break;
            case Launcher::id_vbd_all_in_one: check(ats_vbd_color_sweep(gpu, (int)p.cluster_idx, st), "sweep"); break;
            case Launcher::id_xpbd_read_and_solve_conflict:
                ato_get_x(cpu, buf.data());
                check(ats_async_merge(gpu, buf.data(), 0.5f, st), "merge");
                ++merges;
                break;
            case Launcher::id_xpbd_update_velocity: check(ats_update_velocity(gpu, st), "update"); break;
            default: break;
        }
    };
    auto cpu_dispatch = [&](const Launcher::LaunchParam& p) {
        if (p.function_id == Launcher::id_vbd_all_in_one) ato_vbd_color(cpu, (int)p.cluster_idx);
    };
    const Launcher::Implementation on_gpu(Launcher::DeviceTypeGpu, gpu_dispatch);
    const Launcher::Implementation on_cpu(Launcher::DeviceTypeCpu, cpu_dispatch);
    const std::vector<Launcher::Implementation> g = {on_gpu}, c = {on_cpu};

    Launcher::Scheduler s;
    unsigned prev = s.add_task(Launcher::Task(Launcher::id_xpbd_predict_position, 0, g));
    std::vector<unsigned> order;
    for (int r = 0; r < rounds; ++r) {
        const unsigned fork = s.add_task(Launcher::Task(Launcher::id_xpbd_copy_to_cpu_gpu, (unsigned)r, -1u, 0, g));
        s.set_connect(prev, fork);
        unsigned tail[2] = {fork, fork};
        for (int dev = 0; dev < 2; ++dev)
            for (int it = 0; it < k_iters; ++it)
                for (unsigned col = 0; col < ncol; ++col) {
                    const unsigned t = s.add_task(Launcher::Task(Launcher::id_vbd_all_in_one,
                                                                 (unsigned)(r * k_iters + it), (unsigned)dev, col,
                                                                 dev == 0 ? c : g));
                    s.set_connect(tail[dev], t);
                    tail[dev] = t;
                    order.push_back(t);
                }
        const unsigned merge =
            s.add_task(Launcher::Task(Launcher::id_xpbd_read_and_solve_conflict, (unsigned)r, -1u, 0, g));
        s.set_connect(tail[0], merge);
        s.set_connect(tail[1], merge);
        prev = merge;
    }
    const unsigned last = s.add_task(Launcher::Task(Launcher::id_xpbd_constraint_last_node, 0, g));
    const unsigned upd = s.add_task(Launcher::Task(Launcher::id_xpbd_update_velocity, 0, g));
    s.set_connect(prev, last);
    s.set_connect(last, upd);
    s.set_constraint_task_orders(order);

    std::vector<std::pair<Launcher::FunctionID, unsigned>> keys = {
        {Launcher::id_xpbd_predict_position, 0}, {Launcher::id_xpbd_update_velocity, 0},
        {Launcher::id_xpbd_constraint_last_node, 0}, {Launcher::id_xpbd_copy_to_cpu_gpu, 0},
        {Launcher::id_xpbd_read_and_solve_conflict, 0}};
    for (unsigned col = 0; col < ncol; ++col) keys.push_back({Launcher::id_vbd_all_in_one, col});
    std::vector<std::vector<double>> costs(keys.size(), std::vector<double>{1.0, 1.0});
    std::vector<double> total;
    s.profile_from(keys, costs, total);  // a device without an implementation gets inf
    s.communication_cost_matrix_uma = {{0.0f, 0.1f}, {0.1f, 0.0f}};
    s.communication_speed_matrix = {};
    s.communication_startup = {0.f, 0.f};
    if (!s.topological_sort()) return 3;
    s.standardizing_dag();
    s.scheduler_dag();
    s.make_wait_events();
    s.set_device_stream(Launcher::DeviceTypeGpu, st);
    unsigned on_dev[2] = {0, 0};
    for (const auto& e : s.get_task_schedules())
        if (s.get_list_task()[e.task_id].func_id == Launcher::id_vbd_all_in_one) ++on_dev[e.proc];

    const Launcher::Scheduler::LaunchMode m =
        !std::strcmp(mode, "hetero") ? Launcher::Scheduler::LaunchModeHetero : Launcher::Scheduler::LaunchModeFakeHetero;
    auto to_param = [](const Launcher::Task& t) {
        Launcher::LaunchParam p;
        p.function_id = t.func_id;
        p.iter_idx = t.iter_idx;
        p.cluster_idx = t.cluster_idx;
        p.is_allocated_to_main_device = t.is_allocated_to_main_device;
        return p;
    };
    int status = 0;
    for (int f = 0; f < frames; ++f) {
        check(ats_get_state(gpu, buf.data(), vbuf.data(), st), "state");
        ato_set_state(cpu, buf.data(), vbuf.data());  // the frame start, for the CPU's inertia terms
        ato_frame_begin(cpu);
        s.launch(m, to_param, false);
        status |= (int)s.get_last_launch_status();
        check(ats_frame(alone, ATS_SOLVER_VBD, st), "frame");
    }
    std::vector<float> x(3 * nv), v(3 * nv), xa(3 * nv);
    check(ats_get_state(gpu, x.data(), v.data(), st), "state");
    check(ats_get_state(alone, xa.data(), v.data(), st), "state");
    uint64_t digest = 1469598103934665603ull;
    const unsigned char* b = (const unsigned char*)x.data();
    for (size_t i = 0; i < x.size() * sizeof(float); ++i) digest = (digest ^ b[i]) * 1099511628211ull;
    double dd = 0, nn = 0, disp = 0;
    for (size_t i = 0; i < x.size(); ++i) {
        dd += ((double)x[i] - xa[i]) * ((double)x[i] - xa[i]);
        nn += (double)xa[i] * xa[i];
        disp = std::fmax(disp, std::fabs((double)x[i] - pos[i]));
    }
    std::printf("{\"status\": %d, \"sweeps_on_cpu\": %u, \"sweeps_on_gpu\": %u, \"merges\": %d, \"digest\": \"%016llx\", "
                "\"rel_l2_vs_plain\": %.3e, \"max_displacement\": %.6g, \"cross_device_waits\": %zu}\n",
                status, on_dev[0], on_dev[1], merges, (unsigned long long)digest, std::sqrt(dd / nn), disp,
                s.get_wait_events().size());
    ats_cloth_destroy(gpu);
    ats_cloth_destroy(alone);
    ato_scene_destroy(cpu);
    return 0;
}
