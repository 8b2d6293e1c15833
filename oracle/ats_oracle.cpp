// ats_oracle.cpp -- CPU ORACLE (test infrastructure only).
//
// This file is the checker for the CUDA cloth solver in libatssim_b200. It is a
// plain C++ restatement of libAtsSim's CPU cloth path (ChengzhuUwU/libAtsSim):
// mesh topology, greedy colorings, Vertex Block Descent and XPBD iterations,
// and the energies. Only tests/, __graft_entry__.smoke() and the cpu_baseline /
// reference legs of bench.py load it. The product never links or calls it.
//
// Parity pins (the reference itself cannot be compiled here: it needs glm and a
// Linux TBB, neither installed): the frame-30 sync VBD energy trajectory printed
// in documents/example2_async_convergence.py:78-80 on resources/models/square8K.obj,
// the square8K coloring sizes and the E/B counts of the grid meshes.
//
// Arithmetic follows the reference in FP32 term by term (operation order kept),
// energy sums in FP64 as in parallel_for_and_reduce_sum<double>
// (examples/example2_async_iter.cpp:785-880). Build with -ffp-contract=off so that
// the compiler does not fuse multiply-adds the reference writes separately.
//
// Threading: a std::thread pool with the reference's chunking (256 indices per
// chunk for vertex loops, 32 for per-color loops; src/Utils/cpu_parallel.h:84-99).

#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace ato {

using uint = uint32_t;

// ---------------------------------------------------------------- math types
// Column-major 3-vectors / 3x3 like the reference's Float3 / Float3x3
// (src/SharedDefine/float_n.h, float_n_n.h; get(mat, col, row)).
struct V3 {
    float x, y, z;
};
static inline V3 v3(float a, float b, float c) { return {a, b, c}; }
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct M3 {
    V3 c[3];  // columns
};
static inline M3 m3_zero() { return {{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)}}; }
static inline M3 m3_ident() { return {{v3(1, 0, 0), v3(0, 1, 0), v3(0, 0, 1)}}; }
static inline M3 operator+(const M3& a, const M3& b) { return {{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}}; }
static inline M3 operator-(const M3& a, const M3& b) { return {{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}}; }
static inline M3 operator*(float s, const M3& a) { return {{s * a.c[0], s * a.c[1], s * a.c[2]}}; }
static inline M3 operator*(const M3& a, float s) { return {{a.c[0] * s, a.c[1] * s, a.c[2] * s}}; }
static inline float at(const M3& m, int col, int row) { return comp(m.c[col], row); }
// outer(a, b): column j = a * b_j
static inline M3 outer(V3 a, V3 b) { return {{a * b.x, a * b.y, a * b.z}}; }
// mat * vec = sum_j column_j * v_j
static inline V3 mul(const M3& m, V3 v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }

// 3x3 determinant by cofactor expansion along the first column
// (src/SharedDefine/float_n_n.h:379-385 delegates to the math library).
static inline float det3(const M3& m) {
    return at(m, 0, 0) * (at(m, 1, 1) * at(m, 2, 2) - at(m, 2, 1) * at(m, 1, 2))
         - at(m, 1, 0) * (at(m, 0, 1) * at(m, 2, 2) - at(m, 2, 1) * at(m, 0, 2))
         + at(m, 2, 0) * (at(m, 0, 1) * at(m, 1, 2) - at(m, 1, 1) * at(m, 0, 2));
}
// Adjugate divided element-wise by det (float_n_n.h:283-292 cofactor macros,
// :342-360 inverse_mat(mat, det)).
static inline float cof2(const M3& m, int c1, int c2, int r1, int r2) {
    return at(m, c1, r1) * at(m, c2, r2) - at(m, c1, r2) * at(m, c2, r1);
}
static inline M3 inverse_with_det(const M3& m, float det) {
    M3 o;
    float e[3][3];
    e[0][0] = +cof2(m, 1, 2, 1, 2) / det;
    e[0][1] = -cof2(m, 1, 2, 0, 2) / det;
    e[0][2] = +cof2(m, 1, 2, 0, 1) / det;
    e[1][1] = +cof2(m, 0, 2, 0, 2) / det;
    e[1][2] = -cof2(m, 0, 2, 0, 1) / det;
    e[2][2] = +cof2(m, 0, 1, 0, 1) / det;
    e[1][0] = -cof2(m, 0, 2, 1, 2) / det;
    e[2][0] = +cof2(m, 0, 1, 1, 2) / det;
    e[2][1] = -cof2(m, 0, 1, 0, 2) / det;
    for (int c = 0; c < 3; ++c) o.c[c] = v3(e[c][0], e[c][1], e[c][2]);
    return o;
}

// 4x4, column-major (bending Q).
struct M4 {
    float c[4][4];  // c[col][row]
};

// Hf = [H0 H1 H2 f] (xpbd_constraints.h:4017-4025 makeHf / extractHf)
struct Hf {
    V3 c[4];
};
static inline Hf hf_zero() { return {{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)}}; }
static inline Hf make_hf(V3 f, const M3& h) { return {{h.c[0], h.c[1], h.c[2], f}}; }
static inline Hf& operator+=(Hf& a, const Hf& b) {
    for (int i = 0; i < 4; ++i) a.c[i] += b.c[i];
    return a;
}

static constexpr float kEpsilon = 1.19209290E-7f;  // src/SharedDefine/constant_value.h:9

// ---------------------------------------------------------------- thread pool
class Pool {
public:
    explicit Pool(int n) : nthreads_(std::max(1, n)) {
        for (int i = 1; i < nthreads_; ++i) workers_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    int threads() const { return nthreads_; }
    // Runs fn(i) for i in [0, n) in chunks of `grain` (cpu_parallel.h:84-99).
    void parallel_for(uint n, uint grain, const std::function<void(uint)>& fn) {
        if (n == 0) return;
        if (nthreads_ == 1 || n <= grain) {
            for (uint i = 0; i < n; ++i) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &fn;
            n_ = n;
            grain_ = grain;
            next_.store(0);
            pending_ = nthreads_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

private:
    void work() {
        const std::function<void(uint)>& fn = *job_;
        for (;;) {
            uint b = next_.fetch_add(grain_);
            if (b >= n_) break;
            uint e = std::min(n_, b + grain_);
            for (uint i = b; i < e; ++i) fn(i);
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
            }
            work();
            {
                std::lock_guard<std::mutex> g(mu_);
                if (--pending_ == 0) done_cv_.notify_one();
            }
        }
    }
    int nthreads_;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(uint)>* job_ = nullptr;
    uint n_ = 0, grain_ = 1;
    std::atomic<uint> next_{0};
    int pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// ---------------------------------------------------------------- topology
// Edge and bending-edge extraction: src/Utils/mesh_reader.h:206-298.
// Sort (min, mid, fid), (min, max, fid), (mid, max, fid) triples of every face;
// runs of equal (v0, v1) give one edge (the last of the run, type 0 or 2) and,
// for a pair, one bending edge (v0, v1, opposite of first face, opposite of next).
static void extract_edges(const std::vector<std::array<int, 3>>& faces, std::vector<std::array<int, 2>>& edges,
                          std::vector<std::array<int, 4>>& bending) {
    const size_t nf = faces.size();
    std::vector<std::array<int, 3>> t(nf * 3);
    for (size_t f = 0; f < nf; ++f) {
        int s[3] = {faces[f][0], faces[f][1], faces[f][2]};
        std::sort(s, s + 3);
        t[3 * f + 0] = {s[0], s[1], (int)f};
        t[3 * f + 1] = {s[0], s[2], (int)f};
        t[3 * f + 2] = {s[1], s[2], (int)f};
    }
    std::sort(t.begin(), t.end(), [](const std::array<int, 3>& a, const std::array<int, 3>& b) {
        if (a[0] != b[0]) return a[0] < b[0];
        if (a[1] != b[1]) return a[1] < b[1];
        return a[2] < b[2];
    });
    std::vector<uint8_t> type(t.size(), 0);
    for (size_t i = 0; i < t.size(); ++i) {
        if (i + 1 < t.size() && t[i + 1][0] == t[i][0] && t[i + 1][1] == t[i][1]) type[i] = 1;
        if (i > 0 && t[i - 1][0] == t[i][0] && t[i - 1][1] == t[i][1]) type[i] = 2;
    }
    edges.clear();
    bending.clear();
    for (size_t i = 0; i < t.size(); ++i) {
        if (type[i] == 0 || type[i] == 2) edges.push_back({t[i][0], t[i][1]});
        if (type[i] == 1) {
            const auto& cf = faces[t[i][2]];
            const auto& nf2 = faces[t[i + 1][2]];
            const int a = t[i][0], b = t[i][1];
            const int cr = (cf[0] + cf[1] + cf[2]) - (a + b);
            const int nr = (nf2[0] + nf2[1] + nf2[2]) - (a + b);
            bending.push_back({a, b, cr, nr});
        }
    }
}

// Greedy repeated independent-set extraction in increasing element order:
// examples/example2_async_iter.cpp:458-533 (constraints, nv vertices each)
// and :581-625 (vertices over an adjacency list).
template <typename MarkFn>
static std::vector<std::vector<uint>> greedy_color(uint n, MarkFn mark_neighbours) {
    std::vector<std::vector<uint>> clusters;
    std::vector<uint8_t> marked(n, 0);
    uint total = 0;
    while (true) {
        std::vector<uint> cur;
        std::vector<uint8_t> cur_marked(marked);
        for (uint id = 0; id < n; ++id) {
            if (cur_marked[id]) continue;
            marked[id] = 1;
            cur.push_back(id);
            cur_marked[id] = 1;
            mark_neighbours(id, cur_marked);
        }
        total += (uint)cur.size();
        clusters.push_back(std::move(cur));
        if (total == n) break;
    }
    return clusters;
}

struct Params {
    float implicit_dt;
    int num_substep;
    int iterations;
    float k_stretch;
    float k_bend;  // effective quadratic bending stiffness (after the UI factor)
    float damping;
    float gravity[3];
    int threads;
};

struct Scene {
    Params p;
    std::unique_ptr<Pool> pool;
    uint nv = 0, nf = 0, ne = 0, nb = 0;
    std::vector<V3> rest_x;
    std::vector<std::array<int, 3>> faces;
    std::vector<std::array<int, 2>> edges;
    std::vector<std::array<int, 4>> bending;
    std::vector<float> mass, mass_inv;
    std::vector<uint8_t> fixed;
    std::vector<float> rest_len;
    std::vector<M4> Q;
    // adjacency (example2:229-304)
    std::vector<std::vector<uint>> adj_edges, adj_bending, adj_verts, adj_verts_bending;
    // colorings (example2:442-697)
    std::vector<std::vector<uint>> vert_colors, stretch_colors, bending_colors;
    std::vector<uint> stretch_prefix, bending_prefix;
    std::vector<std::array<int, 2>> merged_edges;
    std::vector<float> merged_rest;
    std::vector<std::array<int, 4>> merged_bending;
    std::vector<M4> merged_Q;
    std::vector<float> lambda_s, lambda_b;
    // state (BasicMeshData / XpbdData, example2:15-88)
    std::vector<V3> x, v, x_start, v_start, x_frame_start, v_frame_start, x_frame_end, v_frame_end;
    std::vector<Hf> hf;
    float sub_dt() const { return p.implicit_dt / float(p.num_substep); }
};

// Rest state: rest length (example2:309-316) and quadratic bending Q
// (example2:344-374; Q = 3/(A0+A1) K K^T from the corner cotangents).
static void init_rest(Scene& s) {
    s.rest_len.resize(s.ne);
    for (uint e = 0; e < s.ne; ++e) {
        V3 a = s.rest_x[s.edges[e][0]], b = s.rest_x[s.edges[e][1]];
        s.rest_len[e] = length(a - b);
    }
    s.Q.resize(s.nb);
    auto cot = [](V3 a, V3 b) { return dot(a, b) / length(cross(a, b)); };
    for (uint e = 0; e < s.nb; ++e) {
        const auto& be = s.bending[e];
        V3 p[4] = {s.rest_x[be[0]], s.rest_x[be[1]], s.rest_x[be[2]], s.rest_x[be[3]]};
        V3 e0 = p[1] - p[0], e1 = p[2] - p[0], e2 = p[3] - p[0], e3 = p[2] - p[1], e4 = p[3] - p[1];
        float c01 = cot(e0, -e1), c02 = cot(e0, -e2), c03 = cot(e0, e3), c04 = cot(e0, e4);
        float K[4] = {c03 + c04, c01 + c02, -c01 - c03, -c02 - c04};
        float A0 = 0.5f * length(cross(e0, e1));
        float A1 = 0.5f * length(cross(e0, e2));
        float sc = 3.f / (A0 + A1);
        M4 q;
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) q.c[c][r] = sc * (K[r] * K[c]);
        s.Q[e] = q;
    }
}

static void init_adjacency(Scene& s) {
    s.adj_edges.assign(s.nv, {});
    s.adj_bending.assign(s.nv, {});
    s.adj_verts.assign(s.nv, {});
    for (uint e = 0; e < s.ne; ++e)
        for (int j = 0; j < 2; ++j) s.adj_edges[s.edges[e][j]].push_back(e);
    for (uint e = 0; e < s.nb; ++e)
        for (int j = 0; j < 4; ++j) s.adj_bending[s.bending[e][j]].push_back(e);
    for (uint e = 0; e < s.ne; ++e)
        for (int j = 0; j < 2; ++j) s.adj_verts[s.edges[e][j]].push_back(s.edges[e][1 - j]);
    s.adj_verts_bending = s.adj_verts;
    for (uint e = 0; e < s.nb; ++e) {
        const auto& be = s.bending[e];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                if (i == j) continue;
                auto& lst = s.adj_verts_bending[be[i]];
                if (std::find(lst.begin(), lst.end(), (uint)be[j]) == lst.end()) lst.push_back(be[j]);
            }
    }
}

static std::vector<uint> prefix_of(const std::vector<std::vector<uint>>& cl) {
    std::vector<uint> p(cl.size() + 1, 0);
    for (size_t c = 0; c < cl.size(); ++c) p[c + 1] = p[c] + (uint)cl[c].size();
    return p;
}

static void init_colorings(Scene& s) {
    s.stretch_colors = greedy_color(s.ne, [&](uint id, std::vector<uint8_t>& m) {
        for (int j = 0; j < 2; ++j)
            for (uint a : s.adj_edges[s.edges[id][j]]) m[a] = 1;
    });
    s.bending_colors = greedy_color(s.nb, [&](uint id, std::vector<uint8_t>& m) {
        for (int j = 0; j < 4; ++j)
            for (uint a : s.adj_bending[s.bending[id][j]]) m[a] = 1;
    });
    s.vert_colors = greedy_color(s.nv, [&](uint id, std::vector<uint8_t>& m) {
        for (uint a : s.adj_verts_bending[id]) m[a] = 1;
    });
    s.stretch_prefix = prefix_of(s.stretch_colors);
    s.bending_prefix = prefix_of(s.bending_colors);
    // colour-merged constraint arrays (example2:648-695)
    s.merged_edges.clear();
    s.merged_rest.clear();
    for (auto& cl : s.stretch_colors)
        for (uint e : cl) {
            s.merged_edges.push_back(s.edges[e]);
            s.merged_rest.push_back(s.rest_len[e]);
        }
    s.merged_bending.clear();
    s.merged_Q.clear();
    for (auto& cl : s.bending_colors)
        for (uint e : cl) {
            s.merged_bending.push_back(s.bending[e]);
            s.merged_Q.push_back(s.Q[e]);
        }
    s.lambda_s.assign(s.ne, 0.f);
    s.lambda_b.assign(s.nb, 0.f);
}

// ---------------------------------------------------------------- solver steps
// Core::predict_position (xpbd_constraints.h:321-384); example2:754-769.
static void predict_position(Scene& s) {
    const float h = s.sub_dt();
    const V3 g = v3(s.p.gravity[0], s.p.gravity[1], s.p.gravity[2]);
    s.pool->parallel_for(s.nv, 256, [&](uint vid) {
        V3 x_prev = s.x_start[vid];
        V3 v_prev = s.v[vid];
        V3 v_pred = v_prev + h * g;
        if (s.fixed[vid]) v_pred = v3(0, 0, 0);
        s.x[vid] = x_prev + h * v_pred;
    });
}

// Core::update_velocity (xpbd_constraints.h:535-581); example2:770-784.
static void update_velocity(Scene& s) {
    const float h = s.sub_dt();
    const float damp = std::exp(-s.p.damping * h);
    s.pool->parallel_for(s.nv, 256, [&](uint vid) {
        V3 xk = s.x[vid];
        V3 dx = xk - s.x_start[vid];
        V3 vel = dx / h;
        vel = vel * damp;
        s.v[vid] = vel;
        s.v_start[vid] = vel;
        s.x_start[vid] = xk;
    });
}

// VBD::compute_inertia (xpbd_constraints.h:4027-4067)
static Hf vbd_inertia(const Scene& s, uint vid, const std::vector<V3>& x) {
    const float h = s.sub_dt();
    const float h2inv = 1.f / (h * h);
    const V3 g = v3(s.p.gravity[0], s.p.gravity[1], s.p.gravity[2]);
    V3 xk = x[vid], x0 = s.x_start[vid], v0 = s.v[vid];
    float m = s.mass[vid];
    M3 mat = (m3_ident() * m) * h2inv;
    V3 outer_force = v3(0, 0, 0);
    outer_force += m * g;
    if (s.fixed[vid]) mat = mat + m3_ident() * float(1e9);
    V3 f = ((-m) * h2inv) * ((xk - x0) - v0 * h) + outer_force;
    return make_hf(f, mat);
}

// VBD::compute_stretch_mass_spring (xpbd_constraints.h:4107-4159)
static Hf vbd_stretch(const Scene& s, uint vid, const std::vector<V3>& x) {
    const float k = s.p.k_stretch;
    Hf hf = hf_zero();
    for (uint e : s.adj_edges[vid]) {
        const auto& ed = s.edges[e];
        V3 p0 = x[ed[0]], p1 = x[ed[1]];
        float L = s.rest_len[e];
        V3 diff = p1 - p0;
        float l = std::max(length(diff), kEpsilon);
        float C = l - L;
        V3 dir = diff / l;
        V3 f0 = (k * dir) * C;
        V3 f1 = -f0;
        M3 xxT = outer(diff, diff);
        float xinv = 1.f / l;
        float xsq = xinv * xinv;
        M3 He = (k * xsq) * xxT + (k * std::max(1.f - L * xinv, 0.f)) * (m3_ident() - xsq * xxT);
        hf += make_hf((uint)ed[0] == vid ? f0 : f1, He);
    }
    return hf;
}

// VBD::compute_bending_quadratic (xpbd_constraints.h:4161-4205)
static Hf vbd_bending(const Scene& s, uint vid, const std::vector<V3>& x) {
    const float kb = s.p.k_bend;
    Hf hf = hf_zero();
    for (uint e : s.adj_bending[vid]) {
        const auto& be = s.bending[e];
        V3 p[4] = {x[be[0]], x[be[1]], x[be[2]], x[be[3]]};
        const M4& Q = s.Q[e];
        int o = (uint)be[0] == vid ? 0 : (uint)be[1] == vid ? 1 : (uint)be[2] == vid ? 2 : 3;
        V3 f = v3(0, 0, 0);
        for (int jj = 0; jj < 4; ++jj) f -= Q.c[o][jj] * p[jj];
        f = f * kb;
        M3 H = (kb * Q.c[o][o]) * m3_ident();
        hf += make_hf(f, H);
    }
    return hf;
}

// One VBD colour (example2:939-1014): inertia, += stretch, += bending, guarded solve.
static void vbd_color(Scene& s, uint c) {
    const auto& cl = s.vert_colors[c];
    const uint n = (uint)cl.size();
    s.pool->parallel_for(n, 256, [&](uint i) { s.hf[cl[i]] = vbd_inertia(s, cl[i], s.x); });
    s.pool->parallel_for(n, 32, [&](uint i) { s.hf[cl[i]] += vbd_stretch(s, cl[i], s.x); });
    s.pool->parallel_for(n, 32, [&](uint i) { s.hf[cl[i]] += vbd_bending(s, cl[i], s.x); });
    s.pool->parallel_for(n, 32, [&](uint i) {
        uint vid = cl[i];
        const Hf& h = s.hf[vid];
        M3 H = {{h.c[0], h.c[1], h.c[2]}};
        V3 f = h.c[3];
        float det = det3(H);
        if (std::fabs(det) > kEpsilon) {
            M3 Hinv = inverse_with_det(H, det);
            s.x[vid] += mul(Hinv, f);
        }
    });
}

// XPBD stretch (xpbd_constraints.h:984-1059), colour loop example2:884-901.
static void xpbd_stretch_color(Scene& s, uint c) {
    const uint b = s.stretch_prefix[c], n = s.stretch_prefix[c + 1] - b;
    const float h = s.sub_dt();
    const float k = s.p.k_stretch;
    s.pool->parallel_for(n, 32, [&](uint i) {
        uint eid = b + i;
        const auto& ed = s.merged_edges[eid];
        float lambda = s.lambda_s[eid];
        V3 p0 = s.x[ed[0]], p1 = s.x[ed[1]];
        float w0 = s.mass_inv[ed[0]], w1 = s.mass_inv[ed[1]];
        float L = s.merged_rest[eid];
        V3 diff = p1 - p0;
        float lsq = dot(diff, diff);
        if (lsq < 1e-8) return;
        float l = std::sqrt(lsq);
        float C = l - L;
        V3 dir = diff / l;
        V3 g1 = -dir;
        float alpha = k < kEpsilon ? 1e9f : 1.f / ((k * h) * h);
        float denom = alpha + (w0 + w1);
        float dl = (-C - alpha * lambda) / denom;
        V3 dx0 = v3(0, 0, 0), dx1 = v3(0, 0, 0);
        if (denom != 0.f) {
            dx0 = (dl * w0) * g1;
            dx1 = ((-dl) * w1) * g1;
        }
        s.lambda_s[eid] = lambda + dl;
        s.x[ed[0]] += dx0;
        s.x[ed[1]] += dx1;
    });
}

// XPBD quadratic bending (xpbd_constraints.h:1062-1126, 1170-1229, 211-236),
// colour loop example2:902-932.
static void xpbd_bending_color(Scene& s, uint c) {
    const uint b = s.bending_prefix[c], n = s.bending_prefix[c + 1] - b;
    const float h = s.sub_dt();
    const float kb = s.p.k_bend;
    s.pool->parallel_for(n, 32, [&](uint i) {
        uint eid = b + i;
        const auto& be = s.merged_bending[eid];
        float w[4];
        V3 p[4];
        for (int j = 0; j < 4; ++j) {
            w[j] = s.mass_inv[be[j]];
            p[j] = s.x[be[j]];
        }
        float lambda = s.lambda_b[eid];
        const M4& Q = s.merged_Q[eid];
        float sum = 0.f;
        for (int ii = 0; ii < 4; ++ii)
            for (int jj = 0; jj < 4; ++jj) sum += Q.c[ii][jj] * dot(p[ii], p[jj]);
        float C = (0.5f * 1.0f) * sum;
        V3 force[4] = {v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)};
        for (int ii = 0; ii < 4; ++ii) {
            for (int jj = 0; jj < 4; ++jj) force[ii] -= Q.c[ii][jj] * p[jj];
            force[ii] = 1.0f * force[ii];
        }
        V3 g[4] = {-force[0], -force[1], -force[2], -force[3]};
        float alpha = kb < kEpsilon ? 1e12f : 1.f / ((kb * h) * h);
        float denom = w[0] * dot(g[0], g[0]) + w[1] * dot(g[1], g[1]) + w[2] * dot(g[2], g[2]) +
                      w[3] * dot(g[3], g[3]) + alpha;
        float dl = (-C - alpha * lambda) / denom;
        V3 dx[4] = {v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0)};
        if (denom != 0.f)
            for (int j = 0; j < 4; ++j) dx[j] = (dl * w[j]) * g[j];
        s.lambda_b[eid] = lambda + dl;
        for (int j = 0; j < 4; ++j) s.x[be[j]] += dx[j];
    });
}

// Energies (xpbd_constraints.h:2079-2214), summed in FP64 as example2:785-880.
static double energy(const Scene& s, const std::vector<V3>& x, bool with_bending) {
    const float h = s.p.implicit_dt / float(s.p.num_substep);
    const V3 g = v3(s.p.gravity[0], s.p.gravity[1], s.p.gravity[2]);
    double ei = 0.0, es = 0.0, eb = 0.0;
    for (uint vid = 0; vid < s.nv; ++vid) {
        V3 a = s.fixed[vid] ? v3(0, 0, 0) : g;
        V3 y = (s.x_start[vid] + h * s.v_start[vid]) + (h * h) * a;
        V3 d = x[vid] - y;
        ei += (double)(dot(d, d) * s.mass[vid] / (2 * h * h));
    }
    for (uint e = 0; e < s.ne; ++e) {
        const auto& ed = s.merged_edges[e];
        V3 diff = x[ed[1]] - x[ed[0]];
        float lsq = dot(diff, diff);
        if (lsq < 1e-8) continue;
        float C = std::sqrt(lsq) - s.merged_rest[e];
        es += (double)(0.5f * s.p.k_stretch * (C * C));
    }
    if (with_bending) {
        for (uint e = 0; e < s.nb; ++e) {
            const auto& be = s.merged_bending[e];
            V3 p[4] = {x[be[0]], x[be[1]], x[be[2]], x[be[3]]};
            const M4& Q = s.merged_Q[e];
            float sum = 0.f;
            for (int ii = 0; ii < 4; ++ii)
                for (int jj = 0; jj < 4; ++jj) sum += Q.c[ii][jj] * dot(p[ii], p[jj]);
            eb += (double)((0.5f * s.p.k_bend) * sum);
        }
    }
    return ei + es + eb;
}

// FP64 incremental-potential gradient norm over free vertices:
// grad_v = m/h^2 (x - y) - f_stretch - f_bending, y = x0 + h v0 + h^2 a.
static double grad_norm(const Scene& s, const std::vector<V3>& x) {
    const double h = (double)s.sub_dt();
    std::vector<double> gr(3 * (size_t)s.nv, 0.0);
    for (uint vid = 0; vid < s.nv; ++vid) {
        const double m = s.mass[vid];
        for (int k = 0; k < 3; ++k) {
            double a = s.fixed[vid] ? 0.0 : (double)s.p.gravity[k];
            double y = (double)comp(s.x_start[vid], k) + h * (double)comp(s.v[vid], k) + h * h * a;
            gr[3 * vid + k] += m / (h * h) * ((double)comp(x[vid], k) - y);
        }
    }
    for (uint e = 0; e < s.ne; ++e) {
        const auto& ed = s.edges[e];
        double d[3], l2 = 0;
        for (int k = 0; k < 3; ++k) {
            d[k] = (double)comp(x[ed[1]], k) - (double)comp(x[ed[0]], k);
            l2 += d[k] * d[k];
        }
        double l = std::sqrt(l2);
        if (l < 1e-30) continue;
        double C = l - (double)s.rest_len[e];
        for (int k = 0; k < 3; ++k) {
            double gk = (double)s.p.k_stretch * C * d[k] / l;  // dE/dx1
            gr[3 * ed[1] + k] += gk;
            gr[3 * ed[0] + k] -= gk;
        }
    }
    // bending gradient k_b sum_j Q_ij (x_j - x_i): the translation-invariant form
    // (every row of Q sums to zero in exact arithmetic)
    for (uint e = 0; e < s.nb; ++e) {
        const auto& be = s.bending[e];
        const M4& Q = s.Q[e];
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k) {
                double acc = 0;
                for (int j = 0; j < 4; ++j)
                    if (j != i) acc += (double)Q.c[i][j] * ((double)comp(x[be[j]], k) - (double)comp(x[be[i]], k));
                gr[3 * be[i] + k] += (double)s.p.k_bend * acc;
            }
    }
    double n2 = 0;
    for (uint vid = 0; vid < s.nv; ++vid)
        if (!s.fixed[vid])
            for (int k = 0; k < 3; ++k) n2 += gr[3 * vid + k] * gr[3 * vid + k];
    return std::sqrt(n2);
}

// The same norm gathered per vertex on the thread pool (each vertex sums its own
// inertia, spring and bending terms over its adjacency lists, then the squares are
// summed in vertex order): the probe of the CPU to-residual frame. It differs from
// grad_norm only in FP64 summation order.
static double grad_norm_pool(const Scene& s, const std::vector<V3>& x) {
    const double h = (double)s.sub_dt();
    std::vector<double> g2(s.nv, 0.0);
    s.pool->parallel_for(s.nv, 256, [&](uint vid) {
        if (s.fixed[vid]) return;
        double gr[3];
        const double m = s.mass[vid];
        for (int k = 0; k < 3; ++k) {
            const double a = (double)s.p.gravity[k];
            const double y = (double)comp(s.x_start[vid], k) + h * (double)comp(s.v[vid], k) + h * h * a;
            gr[k] = m / (h * h) * ((double)comp(x[vid], k) - y);
        }
        for (uint e : s.adj_edges[vid]) {
            const auto& ed = s.edges[e];
            double d[3], l2 = 0;
            for (int k = 0; k < 3; ++k) {
                d[k] = (double)comp(x[ed[1]], k) - (double)comp(x[ed[0]], k);
                l2 += d[k] * d[k];
            }
            const double l = std::sqrt(l2);
            if (l < 1e-30) continue;
            const double C = l - (double)s.rest_len[e];
            const double sign = (uint)ed[1] == vid ? 1.0 : -1.0;
            for (int k = 0; k < 3; ++k) gr[k] += sign * (double)s.p.k_stretch * C * d[k] / l;
        }
        for (uint e : s.adj_bending[vid]) {
            const auto& be = s.bending[e];
            const M4& Q = s.Q[e];
            for (int i = 0; i < 4; ++i) {
                if ((uint)be[i] != vid) continue;
                for (int k = 0; k < 3; ++k) {
                    double acc = 0;
                    for (int j = 0; j < 4; ++j)
                        if (j != i) acc += (double)Q.c[i][j] * ((double)comp(x[be[j]], k) - (double)comp(x[be[i]], k));
                    gr[k] += (double)s.p.k_bend * acc;
                }
            }
        }
        g2[vid] = gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2];
    });
    double n2 = 0;
    for (uint vid = 0; vid < s.nv; ++vid) n2 += g2[vid];
    return std::sqrt(n2);
}

}  // namespace ato

// ---------------------------------------------------------------- C API (ctypes)
using namespace ato;

extern "C" {

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

void* ato_scene_create(const float* pos, int nv, const int* faces, int nf, const float* mass,
                       const unsigned char* fixed, const ato_params* prm) {
    Scene* s = new Scene();
    std::memcpy(&s->p, prm, sizeof(Params));
    s->pool.reset(new Pool(prm->threads));
    s->nv = nv;
    s->nf = nf;
    s->rest_x.resize(nv);
    for (int i = 0; i < nv; ++i) s->rest_x[i] = v3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    s->faces.resize(nf);
    for (int f = 0; f < nf; ++f) s->faces[f] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
    extract_edges(s->faces, s->edges, s->bending);
    s->ne = (uint)s->edges.size();
    s->nb = (uint)s->bending.size();
    s->mass.assign(mass, mass + nv);
    s->fixed.assign(fixed, fixed + nv);
    s->mass_inv.resize(nv);
    for (int i = 0; i < nv; ++i) s->mass_inv[i] = s->fixed[i] ? 0.0f : 1.0f / s->mass[i];
    init_adjacency(*s);
    init_rest(*s);
    init_colorings(*s);
    s->x_frame_start = s->rest_x;
    s->x_frame_end = s->rest_x;
    s->v_frame_start.assign(nv, v3(0, 0, 0));
    s->v_frame_end.assign(nv, v3(0, 0, 0));
    s->x = s->rest_x;
    s->v.assign(nv, v3(0, 0, 0));
    s->x_start = s->rest_x;
    s->v_start.assign(nv, v3(0, 0, 0));
    s->hf.assign(nv, hf_zero());
    return s;
}

void ato_scene_destroy(void* h) { delete (Scene*)h; }

// counts[0..5] = E, B, vertex colours, stretch colours, bending colours, threads
void ato_scene_counts(void* h, int* counts) {
    Scene* s = (Scene*)h;
    counts[0] = (int)s->ne;
    counts[1] = (int)s->nb;
    counts[2] = (int)s->vert_colors.size();
    counts[3] = (int)s->stretch_colors.size();
    counts[4] = (int)s->bending_colors.size();
    counts[5] = s->pool->threads();
}

void ato_get_edges(void* h, int* out) {
    Scene* s = (Scene*)h;
    for (uint e = 0; e < s->ne; ++e) {
        out[2 * e] = s->edges[e][0];
        out[2 * e + 1] = s->edges[e][1];
    }
}
void ato_get_bending(void* h, int* out) {
    Scene* s = (Scene*)h;
    for (uint e = 0; e < s->nb; ++e)
        for (int j = 0; j < 4; ++j) out[4 * e + j] = s->bending[e][j];
}
void ato_get_rest(void* h, float* rest_len, float* q16) {
    Scene* s = (Scene*)h;
    for (uint e = 0; e < s->ne; ++e) rest_len[e] = s->rest_len[e];
    for (uint e = 0; e < s->nb; ++e)
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) q16[16 * e + 4 * c + r] = s->Q[e].c[c][r];
}
// which: 0 vertex colours, 1 stretch colours, 2 bending colours.
// prefix has ncolors+1 entries; items has the element ids in colour order.
void ato_get_coloring(void* h, int which, int* prefix, int* items) {
    Scene* s = (Scene*)h;
    const auto& cl = which == 0 ? s->vert_colors : which == 1 ? s->stretch_colors : s->bending_colors;
    int p = 0;
    for (size_t c = 0; c < cl.size(); ++c) {
        prefix[c] = p;
        for (uint id : cl[c]) items[p++] = (int)id;
    }
    prefix[cl.size()] = p;
}
// adjacency CSR of vert_adj_verts_with_bending (which=0), vert_adj_edges (1),
// vert_adj_bending_edges (2); prefix has nv+1 entries.
int ato_get_adjacency(void* h, int which, int* prefix, int* items) {
    Scene* s = (Scene*)h;
    const auto& a = which == 0 ? s->adj_verts_bending : which == 1 ? s->adj_edges : s->adj_bending;
    int p = 0;
    for (uint v = 0; v < s->nv; ++v) {
        if (prefix) prefix[v] = p;
        for (uint id : a[v]) {
            if (items) items[p] = (int)id;
            ++p;
        }
    }
    if (prefix) prefix[s->nv] = p;
    return p;
}

void ato_set_state(void* h, const float* x, const float* v) {
    Scene* s = (Scene*)h;
    for (uint i = 0; i < s->nv; ++i) {
        s->x_frame_end[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
        s->v_frame_end[i] = v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    }
}
void ato_get_state(void* h, float* x, float* v) {
    Scene* s = (Scene*)h;
    for (uint i = 0; i < s->nv; ++i) {
        x[3 * i] = s->x_frame_end[i].x;
        x[3 * i + 1] = s->x_frame_end[i].y;
        x[3 * i + 2] = s->x_frame_end[i].z;
        v[3 * i] = s->v_frame_end[i].x;
        v[3 * i + 1] = s->v_frame_end[i].y;
        v[3 * i + 2] = s->v_frame_end[i].z;
    }
}
void ato_set_gravity(void* h, float gx, float gy, float gz) {
    Scene* s = (Scene*)h;
    s->p.gravity[0] = gx;
    s->p.gravity[1] = gy;
    s->p.gravity[2] = gz;
}

// One frame: SolverInterface::physics_step + CpuSolver::physics_step_{vbd,xpbd}
// (example2:1615-1648, 1082-1143, 1017-1081). solver 0 = VBD, 1 = XPBD.
// energy_log (nullable) receives iterations+1 values: before iteration 0 and after
// every iteration (print_xpbd_convergence; forces one substep, example2:1100).
// with_bending selects whether the logged energy keeps the bending term (the
// reference's log drops it, example2:832-846). residual_log (nullable) receives
// iterations+1 FP64 gradient norms at the same points.
void ato_frame(void* h, int solver, double* energy_log, int with_bending, double* residual_log) {
    Scene* s = (Scene*)h;
    s->x_frame_start = s->x_frame_end;
    s->v_frame_start = s->v_frame_end;
    s->x_start = s->x_frame_start;
    s->v_start = s->v_frame_start;
    s->x = s->x_frame_start;
    s->v = s->v_frame_start;
    const bool logging = energy_log != nullptr || residual_log != nullptr;
    const int nsub = logging ? 1 : s->p.num_substep;
    int li = 0;
    for (int sub = 0; sub < nsub; ++sub) {
        predict_position(*s);
        if (solver == 1) {
            std::fill(s->lambda_s.begin(), s->lambda_s.end(), 0.f);
            std::fill(s->lambda_b.begin(), s->lambda_b.end(), 0.f);
        }
        for (int it = 0; it < s->p.iterations; ++it) {
            if (logging && it == 0) {
                if (energy_log) energy_log[li] = energy(*s, s->x, with_bending != 0);
                if (residual_log) residual_log[li] = grad_norm(*s, s->x);
                ++li;
            }
            if (solver == 0) {
                for (uint c = 0; c < s->vert_colors.size(); ++c) vbd_color(*s, c);
            } else {
                for (uint c = 0; c < s->stretch_colors.size(); ++c) xpbd_stretch_color(*s, c);
                for (uint c = 0; c < s->bending_colors.size(); ++c) xpbd_bending_color(*s, c);
            }
            if (logging) {
                if (energy_log) energy_log[li] = energy(*s, s->x, with_bending != 0);
                if (residual_log) residual_log[li] = grad_norm(*s, s->x);
                ++li;
            }
        }
        update_velocity(*s);
    }
    s->x_frame_end = s->x;
    s->v_frame_end = s->v;
}

// One VBD frame iterated to a relative residual, the CPU counterpart of the GPU's
// residual-driven frame (the reference defines no residual; it is the norm of the
// incremental-potential gradient over free vertices, relative to its value at the
// inertial prediction y). Per substep: predict; r0 = ||grad G(y)||; VBD iterations
// (example2:1481-1509) with probes; the substep stops once ||grad G(x)|| <= tol * r0 (or
// at once when r0 == 0) or at max_iterations; then the velocity update. Probes:
// policy 0 after every check_every iterations and at max_iterations; policy 1 (the
// GPU's extrapolated schedule) the first two as policy 0, then after half of the
// iterations that the contraction per iteration between the last two probes predicts
// are still needed (at least check_every, rounded up to a multiple of it), or at
// max_iterations when the residual did not fall. Returns the iterations of the last
// substep; *rel_out (nullable) receives its last probed relative residual.
int ato_frame_to_residual(void* h, double tol, int check_every, int max_iterations, int policy, double* rel_out) {
    Scene* s = (Scene*)h;
    s->x_frame_start = s->x_frame_end;
    s->v_frame_start = s->v_frame_end;
    s->x_start = s->x_frame_start;
    s->v_start = s->v_frame_start;
    s->x = s->x_frame_start;
    s->v = s->v_frame_start;
    if (check_every < 1) check_every = 1;
    int used = 0;
    double rel = 0.0;
    for (int sub = 0; sub < s->p.num_substep; ++sub) {
        predict_position(*s);
        const double r0 = grad_norm_pool(*s, s->x);
        used = 0;
        rel = r0 > 0.0 ? 1.0 : 0.0;
        int next_due = check_every, last_it = 0;
        double last_res = 1.0;
        while (r0 > 0.0 && used < max_iterations) {
            const int target = std::min(policy == 1 ? next_due : used + check_every, max_iterations);
            for (; used < target; ++used)
                for (uint c = 0; c < s->vert_colors.size(); ++c) vbd_color(*s, c);
            rel = grad_norm_pool(*s, s->x) / r0;
            if (rel <= tol || used >= max_iterations) break;
            if (policy == 1) {
                int gap = check_every;
                if (last_it > 0) {
                    gap = max_iterations - used;
                    if (rel < last_res && rel > 0.0 && tol > 0.0) {
                        const double rho = std::pow(rel / last_res, 1.0 / (double)(used - last_it));
                        const double need = std::log(tol / rel) / std::log(rho);
                        if (need < (double)(max_iterations - used)) {
                            const int half = (int)std::ceil(0.5 * need);
                            gap = ((std::max(half, check_every) + check_every - 1) / check_every) * check_every;
                        }
                    }
                }
                next_due = std::min(used + gap, max_iterations);
                last_it = used;
                last_res = rel;
            }
        }
        update_velocity(*s);
    }
    s->x_frame_end = s->x;
    s->v_frame_end = s->v;
    if (rel_out) *rel_out = rel;
    return used;
}

// The frame as separate steps, for a scheduler that runs each task on its own
// device: ato_frame_begin (the frame-start bookkeeping of ato_frame), ato_predict
// (Core::predict_position), ato_vbd_color (one colour of solve_constraints_VBD),
// ato_update (Core::update_velocity, then the frame-end state), and access to the
// current iterate x (3 floats per vertex).
void ato_frame_begin(void* h) {
    Scene* s = (Scene*)h;
    s->x_frame_start = s->x_frame_end;
    s->v_frame_start = s->v_frame_end;
    s->x_start = s->x_frame_start;
    s->v_start = s->v_frame_start;
    s->x = s->x_frame_start;
    s->v = s->v_frame_start;
}
void ato_predict(void* h) { predict_position(*(Scene*)h); }
void ato_vbd_color(void* h, int c) {
    Scene* s = (Scene*)h;
    if (c >= 0 && (size_t)c < s->vert_colors.size()) vbd_color(*s, (uint)c);
}
void ato_update(void* h) {
    Scene* s = (Scene*)h;
    update_velocity(*s);
    s->x_frame_end = s->x;
    s->v_frame_end = s->v;
}
void ato_get_x(void* h, float* x) {
    Scene* s = (Scene*)h;
    for (uint i = 0; i < s->nv; ++i) {
        x[3 * i] = s->x[i].x;
        x[3 * i + 1] = s->x[i].y;
        x[3 * i + 2] = s->x[i].z;
    }
}
void ato_set_x(void* h, const float* x) {
    Scene* s = (Scene*)h;
    for (uint i = 0; i < s->nv; ++i) s->x[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
}

// Runs `frames` frames back to back (no logging), for the CPU baseline timing.
void ato_run_frames(void* h, int solver, int frames) {
    for (int f = 0; f < frames; ++f) ato_frame(h, solver, nullptr, 0, nullptr);
}

// Energy / gradient norm of an arbitrary position array against the current
// frame-start state (x_start, v_start), FP64.
double ato_energy_of(void* h, const float* xin, int with_bending) {
    Scene* s = (Scene*)h;
    std::vector<V3> x(s->nv);
    for (uint i = 0; i < s->nv; ++i) x[i] = v3(xin[3 * i], xin[3 * i + 1], xin[3 * i + 2]);
    return energy(*s, x, with_bending != 0);
}
double ato_grad_norm_of(void* h, const float* xin) {
    Scene* s = (Scene*)h;
    std::vector<V3> x(s->nv);
    for (uint i = 0; i < s->nv; ++i) x[i] = v3(xin[3 * i], xin[3 * i + 1], xin[3 * i + 2]);
    return grad_norm(*s, x);
}
double ato_grad_norm_pool_of(void* h, const float* xin) {
    Scene* s = (Scene*)h;
    std::vector<V3> x(s->nv);
    for (uint i = 0; i < s->nv; ++i) x[i] = v3(xin[3 * i], xin[3 * i + 1], xin[3 * i + 2]);
    return grad_norm_pool(*s, x);
}
// Prepare a frame for energy_of / grad_norm_of: x_start = frame end state, v = frame end v.
void ato_begin_frame(void* h) {
    Scene* s = (Scene*)h;
    s->x_start = s->x_frame_end;
    s->v_start = s->v_frame_end;
    s->v = s->v_frame_end;
}

// Reference rules for pins and mass (example2:185-225).
void ato_reference_pins(const float* pos, int nv, unsigned char* fixed) {
    float mn[3] = {pos[0], pos[1], pos[2]}, mx[3] = {pos[0], pos[1], pos[2]};
    for (int i = 1; i < nv; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], pos[3 * i + k]);
            mx[k] = std::max(mx[k], pos[3 * i + k]);
        }
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / std::max(kEpsilon, mx[k] - mn[k]);  // AABB::range_inv (aabb.h:70-75)
    for (int i = 0; i < nv; ++i) {
        float nx = (pos[3 * i + 0] - mn[0]) * inv[0];
        float nz = (pos[3 * i + 2] - mn[2]) * inv[2];
        fixed[i] = (nz < 0.01f && (nx > 0.99f || nx < 0.01f)) ? 1 : 0;
    }
}

}  // extern "C"
