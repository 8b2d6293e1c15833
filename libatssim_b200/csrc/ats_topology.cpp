// ats_topology.cpp -- host topology, mesh helpers and the colour-major device layout.
// Compiled with -ffp-contract=off: the float rest state (lengths, Q) is computed
// term by term as examples/example2_async_iter.cpp:309-375 writes it.

#include "ats_topology.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace ats {

namespace {

struct F3 {
    float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 neg(F3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len(F3 a) { return std::sqrt(dot(a, a)); }
inline F3 at(const std::vector<float>& p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

// Greedy colouring: repeatedly sweep the elements in increasing id and take every
// element not yet coloured and not touched in this sweep; touching marks the
// neighbours given by `neighbours(id, mark)`. Equivalent to the copy-the-mask loop
// of example2_async_iter.cpp:458-533 / :581-625 (a sweep stamp replaces the copy).
template <typename Neighbours>
void greedy_colour(int n, Neighbours neighbours, std::vector<int>& off, std::vector<int>& items) {
    std::vector<uint8_t> done(n, 0);
    std::vector<int> stamp(n, -1);
    off.assign(1, 0);
    items.clear();
    items.reserve(n);
    int coloured = 0;
    for (int sweep = 0;; ++sweep) {
        auto mark = [&](int id) { stamp[id] = sweep; };
        for (int id = 0; id < n; ++id) {
            if (done[id] || stamp[id] == sweep) continue;
            done[id] = 1;
            stamp[id] = sweep;
            items.push_back(id);
            ++coloured;
            neighbours(id, mark);
        }
        off.push_back((int)items.size());
        if (coloured == n) break;
    }
}

void build_csr(int nv, const std::vector<int>& elems, int per, std::vector<int>& off, std::vector<int>& items) {
    const int n = (int)elems.size() / per;
    off.assign(nv + 1, 0);
    for (int e = 0; e < n; ++e)
        for (int j = 0; j < per; ++j) off[elems[per * e + j] + 1]++;
    for (int v = 0; v < nv; ++v) off[v + 1] += off[v];
    items.assign(off[nv], 0);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int e = 0; e < n; ++e)
        for (int j = 0; j < per; ++j) items[fill[elems[per * e + j]]++] = e;
}

}  // namespace

bool build_topology(const ats_instance_desc& d, Topology& t, std::string& err) {
    if (d.num_verts <= 0 || d.num_faces < 0 || !d.positions || (d.num_faces > 0 && !d.faces)) {
        err = "mesh needs num_verts > 0, positions and faces";
        return false;
    }
    t = Topology();
    t.nv = d.num_verts;
    t.pos.assign(d.positions, d.positions + 3 * (size_t)d.num_verts);
    t.faces.reserve(3 * (size_t)d.num_faces);
    for (int f = 0; f < d.num_faces; ++f) {
        int a = d.faces[3 * f], b = d.faces[3 * f + 1], c = d.faces[3 * f + 2];
        if (a < 0 || b < 0 || c < 0 || a >= t.nv || b >= t.nv || c >= t.nv) {
            err = "face " + std::to_string(f) + " has a vertex index out of range";
            return false;
        }
        if (a == b || a == c || b == c) continue;  // mesh_reader.cpp:170-177 drops degenerate faces
        t.faces.push_back(a);
        t.faces.push_back(b);
        t.faces.push_back(c);
    }
    t.nf = (int)t.faces.size() / 3;

    // ---- edges and bending edges (mesh_reader.h:206-298)
    struct Rec {
        int a, b, f;
    };
    std::vector<Rec> r(3 * (size_t)t.nf);
    for (int f = 0; f < t.nf; ++f) {
        int s[3] = {t.faces[3 * f], t.faces[3 * f + 1], t.faces[3 * f + 2]};
        std::sort(s, s + 3);
        r[3 * f + 0] = {s[0], s[1], f};
        r[3 * f + 1] = {s[0], s[2], f};
        r[3 * f + 2] = {s[1], s[2], f};
    }
    std::sort(r.begin(), r.end(), [](const Rec& x, const Rec& y) {
        if (x.a != y.a) return x.a < y.a;
        if (x.b != y.b) return x.b < y.b;
        return x.f < y.f;
    });
    const size_t nr = r.size();
    auto same = [&](size_t i, size_t j) { return r[i].a == r[j].a && r[i].b == r[j].b; };
    for (size_t i = 0; i < nr; ++i) {
        // type: 0 boundary, 1 first of a shared pair, 2 later member of a run
        int type = 0;
        if (i + 1 < nr && same(i, i + 1)) type = 1;
        if (i > 0 && same(i, i - 1)) type = 2;
        if (type != 1) {
            t.edges.push_back(r[i].a);
            t.edges.push_back(r[i].b);
        } else {
            const int a = r[i].a, b = r[i].b;
            const int* f0 = &t.faces[3 * r[i].f];
            const int* f1 = &t.faces[3 * r[i + 1].f];
            t.bending.push_back(a);
            t.bending.push_back(b);
            t.bending.push_back((f0[0] + f0[1] + f0[2]) - (a + b));
            t.bending.push_back((f1[0] + f1[1] + f1[2]) - (a + b));
        }
    }
    const int ne = (int)t.edges.size() / 2, nb = (int)t.bending.size() / 4;

    // ---- adjacency (example2_async_iter.cpp:229-304)
    build_csr(t.nv, t.edges, 2, t.ve_off, t.ve);
    build_csr(t.nv, t.bending, 4, t.vb_off, t.vb);

    // ---- rest state (example2_async_iter.cpp:309-375)
    t.rest.resize(ne);
    for (int e = 0; e < ne; ++e) t.rest[e] = len(sub(at(t.pos, t.edges[2 * e]), at(t.pos, t.edges[2 * e + 1])));
    t.q.assign(16 * (size_t)nb, 0.f);
    auto cot = [](F3 a, F3 b) { return dot(a, b) / len(cross(a, b)); };
    for (int e = 0; e < nb; ++e) {
        const int* be = &t.bending[4 * e];
        F3 p0 = at(t.pos, be[0]), p1 = at(t.pos, be[1]), p2 = at(t.pos, be[2]), p3 = at(t.pos, be[3]);
        F3 e0 = sub(p1, p0), e1 = sub(p2, p0), e2 = sub(p3, p0), e3 = sub(p2, p1), e4 = sub(p3, p1);
        float c01 = cot(e0, neg(e1)), c02 = cot(e0, neg(e2)), c03 = cot(e0, e3), c04 = cot(e0, e4);
        float K[4] = {c03 + c04, c01 + c02, -c01 - c03, -c02 - c04};
        float A0 = 0.5f * len(cross(e0, e1));
        float A1 = 0.5f * len(cross(e0, e2));
        float sc = 3.f / (A0 + A1);
        for (int c = 0; c < 4; ++c)
            for (int rr = 0; rr < 4; ++rr) t.q[16 * (size_t)e + 4 * c + rr] = sc * (K[rr] * K[c]);
    }

    // ---- colourings
    greedy_colour(
        ne,
        [&](int id, auto& mark) {
            for (int j = 0; j < 2; ++j) {
                int v = t.edges[2 * id + j];
                for (int k = t.ve_off[v]; k < t.ve_off[v + 1]; ++k) mark(t.ve[k]);
            }
        },
        t.scol_off, t.scol);
    greedy_colour(
        nb,
        [&](int id, auto& mark) {
            for (int j = 0; j < 4; ++j) {
                int v = t.bending[4 * id + j];
                for (int k = t.vb_off[v]; k < t.vb_off[v + 1]; ++k) mark(t.vb[k]);
            }
        },
        t.bcol_off, t.bcol);
    // vertex neighbours = edge neighbours plus the other corners of adjacent bending
    // edges (vert_adj_verts_with_bending); only membership matters for the colouring.
    greedy_colour(
        t.nv,
        [&](int v, auto& mark) {
            for (int k = t.ve_off[v]; k < t.ve_off[v + 1]; ++k) {
                int e = t.ve[k];
                mark(t.edges[2 * e] == v ? t.edges[2 * e + 1] : t.edges[2 * e]);
            }
            for (int k = t.vb_off[v]; k < t.vb_off[v + 1]; ++k) {
                const int* be = &t.bending[4 * t.vb[k]];
                for (int j = 0; j < 4; ++j)
                    if (be[j] != v) mark(be[j]);
            }
        },
        t.vcol_off, t.vcol);
    return true;
}

bool build_slices(Layout& L, int tpv, std::string& err) {
    if (tpv != 1 && tpv != 2 && tpv != 4 && tpv != 8) {
        err = "threads_per_vertex must be 1, 2, 4 or 8";
        return false;
    }
    L.tpv = tpv;
    const int vps = 32 / tpv;  // vertices per slice (one warp)
    // size the arrays first
    size_t total = 0;
    size_t nslices = 0;
    auto slice_rows = [&](int s, int n, int& erows, int& brows) {
        int max_e = 0, max_b = 0;
        for (int k = 0; k < n; ++k) {
            const int ne = L.nb_nedge[s + k];
            max_e = std::max(max_e, ne);
            max_b = std::max(max_b, L.nb_off[s + k + 1] - L.nb_off[s + k] - ne);
        }
        erows = (max_e + tpv - 1) / tpv;
        brows = (max_b + tpv - 1) / tpv;
    };
    for (int c = 0; c < L.n_vcolors; ++c)
        for (int ri = L.run_off[c]; ri < L.run_off[c + 1]; ++ri)
            for (int s = L.runs[2 * ri]; s < L.runs[2 * ri + 1]; s += vps) {
                int er, br;
                slice_rows(s, std::min(vps, L.runs[2 * ri + 1] - s), er, br);
                total += 32 * (size_t)(er + br);
                ++nslices;
            }
    L.st_iw.assign(2 * total, 0);
    L.st_rest.assign(total, -1.f);
    L.slices.clear();
    L.slices.reserve(4 * nslices);
    L.color_slices.assign(1, 0);
    size_t off = 0;
    // entry (row, thread th) of a slice = vertex th / tpv, slot row * tpv + th % tpv
    // within the edge rows (first erows rows) or the bending-only rows
    for (int c = 0; c < L.n_vcolors; ++c) {
        for (int ri = L.run_off[c]; ri < L.run_off[c + 1]; ++ri) {
            const int b = L.runs[2 * ri], e = L.runs[2 * ri + 1];
            for (int s = b; s < e; s += vps) {
                const int n = std::min(vps, e - s);
                int erows, brows;
                slice_rows(s, n, erows, brows);
                const int rows = erows + brows;
                for (int th = 0; th < 32; ++th) {
                    const int k = th / tpv;
                    const int self = s + std::min(k, n - 1);
                    const int lo = k < n ? L.nb_off[s + k] : 0;
                    const int ne = k < n ? L.nb_nedge[s + k] : 0;
                    const int nb = k < n ? L.nb_off[s + k + 1] - lo - ne : 0;
                    for (int row = 0; row < rows; ++row) {
                        const bool edge_row = row < erows;
                        const int slot = (edge_row ? row : row - erows) * tpv + th % tpv;
                        const size_t at = off + 32 * (size_t)row + th;
                        int idx = self;
                        float w = 0.f, rest = -1.f;
                        if (edge_row ? slot < ne : slot < nb) {
                            const int q = lo + (edge_row ? slot : ne + slot);
                            idx = L.nb_u[q];
                            w = L.nb_w[q];
                            rest = edge_row ? L.nb_rest[q] : -1.f;
                        }
                        L.st_iw[2 * at] = idx;
                        std::memcpy(&L.st_iw[2 * at + 1], &w, 4);
                        L.st_rest[at] = rest;
                    }
                }
                L.slices.push_back(s);
                L.slices.push_back(n);
                L.slices.push_back((int)off);
                L.slices.push_back(rows | (erows << 16));
                off += 32 * (size_t)rows;
            }
        }
        L.color_slices.push_back((int)L.slices.size() / 4);
    }
    return true;
}

bool build_layout(const std::vector<Topology>& topos, const std::vector<ats_instance_desc>& descs, const float* gravity,
                  int tpv, Layout& L, std::string& err) {
    L = Layout();
    L.ninst = (int)topos.size();
    L.inst_vbegin.assign(1, 0);
    for (const auto& t : topos) {
        L.nv += t.nv;
        L.ne += t.ne();
        L.nb += t.nb();
        L.n_vcolors = std::max(L.n_vcolors, t.nvc());
        L.n_scolors = std::max(L.n_scolors, t.nsc());
        L.n_bcolors = std::max(L.n_bcolors, t.nbc());
        L.inst_vbegin.push_back(L.nv);
    }
    L.to_layout.assign(L.nv, -1);
    L.to_caller.assign(L.nv, -1);
    L.x0.assign(4 * (size_t)L.nv, 0.f);
    L.vel.assign(4 * (size_t)L.nv, 0.f);
    L.vm.assign(4 * (size_t)L.nv, 0.f);
    L.inst.assign(4 * (size_t)L.ninst, 0.f);
    for (int i = 0; i < L.ninst; ++i) {
        for (int k = 0; k < 3; ++k) L.inst[4 * i + k] = gravity[k];
        L.inst[4 * i + 3] = descs[i].k_stretch;
    }

    // vertex order: instance-major, colour-major, increasing vertex id in a colour
    std::vector<std::vector<int>> inst_colour_begin(L.ninst);  // layout id where colour c starts
    for (int i = 0; i < L.ninst; ++i) {
        const Topology& t = topos[i];
        int p = L.inst_vbegin[i];
        for (int c = 0; c < t.nvc(); ++c) {
            inst_colour_begin[i].push_back(p);
            for (int k = t.vcol_off[c]; k < t.vcol_off[c + 1]; ++k) {
                int orig = L.inst_vbegin[i] + t.vcol[k];
                L.to_layout[orig] = p;
                L.to_caller[p] = orig;
                ++p;
            }
        }
        inst_colour_begin[i].push_back(p);
        if (p != L.inst_vbegin[i + 1]) {
            err = "vertex colouring does not cover every vertex";
            return false;
        }
    }
    L.run_off.assign(1, 0);
    for (int c = 0; c < L.n_vcolors; ++c) {
        for (int i = 0; i < L.ninst; ++i) {
            if (c >= topos[i].nvc()) continue;
            int b = inst_colour_begin[i][c], e = inst_colour_begin[i][c + 1];
            if (e > b) {
                L.runs.push_back(b);
                L.runs.push_back(e);
            }
        }
        L.run_off.push_back((int)L.runs.size() / 2);
    }

    // per-vertex data and neighbour lists (in layout ids): edge neighbours first,
    // then bending-only neighbours, each sorted by id; bending weights summed in FP64
    struct Nb {
        int u;
        float rest;
        double w;
    };
    std::vector<std::vector<Nb>> sten(L.nv);
    std::vector<int> nedge(L.nv, 0);
    for (int i = 0; i < L.ninst; ++i) {
        const Topology& t = topos[i];
        const ats_instance_desc& d = descs[i];
        const int ob = L.inst_vbegin[i];
        std::vector<Nb> cand;
        for (int v = 0; v < t.nv; ++v) {
            const int lv = L.to_layout[ob + v];
            cand.clear();
            for (int k = t.ve_off[v]; k < t.ve_off[v + 1]; ++k) {
                const int e = t.ve[k];
                const int u = t.edges[2 * e] == v ? t.edges[2 * e + 1] : t.edges[2 * e];
                cand.push_back(Nb{L.to_layout[ob + u], t.rest[e], 0.0});
            }
            double hdiag = 0.0;
            for (int k = t.vb_off[v]; k < t.vb_off[v + 1]; ++k) {
                const int e = t.vb[k];
                const int* be = &t.bending[4 * e];
                const int o = be[0] == v ? 0 : be[1] == v ? 1 : be[2] == v ? 2 : 3;
                const float* Q = &t.q[16 * (size_t)e];  // Q[col][row], symmetric
                hdiag += (double)Q[4 * o + o];
                for (int j = 0; j < 4; ++j)
                    if (j != o) cand.push_back(Nb{L.to_layout[ob + be[j]], -2.f, (double)Q[4 * o + j]});
            }
            // merge by neighbour id: the edge entry carries the rest length
            std::sort(cand.begin(), cand.end(), [](const Nb& x, const Nb& y) { return x.u < y.u; });
            std::vector<Nb>& out = sten[lv];
            for (size_t k = 0; k < cand.size();) {
                Nb m{cand[k].u, -1.f, 0.0};
                size_t j = k;
                for (; j < cand.size() && cand[j].u == m.u; ++j) {
                    if (cand[j].rest > -2.f) m.rest = cand[j].rest;
                    m.w += cand[j].w;
                }
                out.push_back(m);
                k = j;
            }
            std::stable_partition(out.begin(), out.end(), [](const Nb& x) { return x.rest >= 0.f; });
            for (const Nb& x : out) nedge[lv] += x.rest >= 0.f;
            const double kb = d.k_bend;
            for (Nb& x : out) x.w *= kb;
            const float mass = d.mass[v];
            const bool fixed = d.fixed[v] != 0;
            L.x0[4 * (size_t)lv + 0] = t.pos[3 * v];
            L.x0[4 * (size_t)lv + 1] = t.pos[3 * v + 1];
            L.x0[4 * (size_t)lv + 2] = t.pos[3 * v + 2];
            L.x0[4 * (size_t)lv + 3] = mass;
            L.vm[4 * (size_t)lv + 0] = (float)(kb * hdiag);
            L.vel[4 * (size_t)lv + 3] = L.vm[4 * (size_t)lv + 0];  // for the list sweep, which skips vm
            L.vm[4 * (size_t)lv + 1] = fixed ? 1e9f : 0.f;
            L.vm[4 * (size_t)lv + 2] = fixed ? 0.f : 1.0f / mass;
            int inst_id = i;
            std::memcpy(&L.vm[4 * (size_t)lv + 3], &inst_id, 4);
        }
    }
    L.nb_off.assign(1, 0);
    L.nb_nedge = nedge;
    for (int lv = 0; lv < L.nv; ++lv) {
        for (const Nb& nb : sten[lv]) {
            L.nb_u.push_back(nb.u);
            L.nb_rest.push_back(nb.rest);
            L.nb_w.push_back((float)nb.w);
        }
        L.nb_off.push_back((int)L.nb_u.size());
    }
    sten.clear();
    if (!build_slices(L, tpv, err)) return false;

    // XPBD constraints, colour-major over instances (example2_async_iter.cpp:648-695)
    L.xs_color.assign(1, 0);
    for (int c = 0; c < L.n_scolors; ++c) {
        for (int i = 0; i < L.ninst; ++i) {
            const Topology& t = topos[i];
            if (c >= t.nsc()) continue;
            const int ob = L.inst_vbegin[i];
            for (int k = t.scol_off[c]; k < t.scol_off[c + 1]; ++k) {
                int e = t.scol[k];
                L.xs_edge.push_back(L.to_layout[ob + t.edges[2 * e]]);
                L.xs_edge.push_back(L.to_layout[ob + t.edges[2 * e + 1]]);
                L.xs_rest.push_back(t.rest[e]);
                L.xs_k.push_back(descs[i].k_stretch);
            }
        }
        L.xs_color.push_back((int)L.xs_rest.size());
    }
    L.xb_color.assign(1, 0);
    for (int c = 0; c < L.n_bcolors; ++c) {
        for (int i = 0; i < L.ninst; ++i) {
            const Topology& t = topos[i];
            if (c >= t.nbc()) continue;
            const int ob = L.inst_vbegin[i];
            for (int k = t.bcol_off[c]; k < t.bcol_off[c + 1]; ++k) {
                int e = t.bcol[k];
                for (int j = 0; j < 4; ++j) L.xb_idx.push_back(L.to_layout[ob + t.bending[4 * e + j]]);
                const float* Q = &t.q[16 * (size_t)e];
                const int uc[10][2] = {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {1, 1}, {1, 2}, {1, 3}, {2, 2}, {2, 3}, {3, 3}};
                for (auto& p : uc) L.xb_q.push_back(Q[4 * p[0] + p[1]]);
                L.xb_q.push_back(descs[i].k_bend);
                L.xb_q.push_back(0.f);
            }
        }
        L.xb_color.push_back((int)L.xb_idx.size() / 4);
    }

    // energy terms in original element order, instance by instance
    L.inst_eseg.assign(1, 0);
    L.inst_bseg.assign(1, 0);
    for (int i = 0; i < L.ninst; ++i) {
        const Topology& t = topos[i];
        const int ob = L.inst_vbegin[i];
        for (int e = 0; e < t.ne(); ++e) {
            L.en_edge.push_back(L.to_layout[ob + t.edges[2 * e]]);
            L.en_edge.push_back(L.to_layout[ob + t.edges[2 * e + 1]]);
            L.en_rest.push_back(t.rest[e]);
            L.en_k.push_back(descs[i].k_stretch);
        }
        for (int e = 0; e < t.nb(); ++e) {
            for (int j = 0; j < 4; ++j) L.en_bend.push_back(L.to_layout[ob + t.bending[4 * e + j]]);
            for (int j = 0; j < 16; ++j) L.en_q.push_back(t.q[16 * (size_t)e + j]);
            L.en_kb.push_back(descs[i].k_bend);
        }
        L.inst_eseg.push_back((int)L.en_rest.size());
        L.inst_bseg.push_back((int)L.en_kb.size());
    }

    // direction slots of the edge neighbours (rest plane x-z): the six neighbour
    // directions of a uniform-diagonal grid vertex, nearest angle wins
    static const double kSlotDeg[6] = {0.0, 45.0, 90.0, 180.0, 225.0, 270.0};
    L.feat_nb.assign(6 * (size_t)L.nv, -1);
    L.feat_len.assign(6 * (size_t)L.nv, 0.f);
    std::vector<double> best(6);
    for (int i = 0; i < L.ninst; ++i) {
        const Topology& t = topos[i];
        const int ob = L.inst_vbegin[i];
        for (int v = 0; v < t.nv; ++v) {
            const int lv = L.to_layout[ob + v];
            std::fill(best.begin(), best.end(), 1e30);
            for (int k = t.ve_off[v]; k < t.ve_off[v + 1]; ++k) {
                const int e = t.ve[k];
                const int u = t.edges[2 * e] == v ? t.edges[2 * e + 1] : t.edges[2 * e];
                const double dx = (double)t.pos[3 * u] - t.pos[3 * v], dz = (double)t.pos[3 * u + 2] - t.pos[3 * v + 2];
                double deg = std::atan2(dz, dx) * 57.29577951308232;
                if (deg < 0) deg += 360.0;
                int slot = 0;
                double dist = 1e30;
                for (int q = 0; q < 6; ++q) {
                    double d = std::fabs(deg - kSlotDeg[q]);
                    d = std::min(d, 360.0 - d);
                    if (d < dist) {
                        dist = d;
                        slot = q;
                    }
                }
                if (dist < best[slot]) {
                    best[slot] = dist;
                    L.feat_nb[6 * (size_t)lv + slot] = L.to_layout[ob + u];
                    L.feat_len[6 * (size_t)lv + slot] = t.rest[e];
                }
            }
        }
    }
    return true;
}

}  // namespace ats

// ---------------------------------------------------------------- C ABI (host only)
using namespace ats;

namespace ats {
void set_error(const std::string& msg);
}

struct ats_topology {
    Topology t;
};

extern "C" {

int ats_grid_mesh(int n, int pattern, float* positions, int* faces) {
    if (n < 2 || !positions || !faces || (pattern != ATS_GRID_UNIFORM && pattern != ATS_GRID_ALTERNATING)) {
        set_error("ats_grid_mesh: need n >= 2, output arrays and a known pattern");
        return ATS_ERR_INVALID;
    }
    const float inv = 1.0f / float(n - 1);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            float* p = positions + 3 * ((size_t)r * n + c);
            p[0] = -0.5f + float(c) * inv;
            p[1] = 0.f;
            p[2] = -0.5f + float(r) * inv;
        }
    size_t k = 0;
    for (int r = 0; r < n - 1; ++r)
        for (int c = 0; c < n - 1; ++c) {
            int a = r * n + c, b = a + 1, d = a + n, e = d + 1;
            bool even = ((r + c) % 2) == 0;
            if (pattern == ATS_GRID_UNIFORM || even) {
                int tri[6] = {a, e, b, a, d, e};
                for (int j = 0; j < 6; ++j) faces[k++] = tri[j];
            } else {
                int tri[6] = {a, d, b, b, d, e};
                for (int j = 0; j < 6; ++j) faces[k++] = tri[j];
            }
        }
    return ATS_OK;
}

int ats_reference_pins(const float* pos, int nv, unsigned char* fixed) {
    if (!pos || !fixed || nv <= 0) {
        set_error("ats_reference_pins: bad arguments");
        return ATS_ERR_INVALID;
    }
    const float eps = 1.19209290E-7f;
    float mn[3] = {pos[0], pos[1], pos[2]}, mx[3] = {pos[0], pos[1], pos[2]};
    for (int i = 1; i < nv; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], pos[3 * i + k]);
            mx[k] = std::max(mx[k], pos[3 * i + k]);
        }
    float inv[3];
    for (int k = 0; k < 3; ++k) inv[k] = 1.0f / std::max(eps, mx[k] - mn[k]);
    for (int i = 0; i < nv; ++i) {
        float nx = (pos[3 * i] - mn[0]) * inv[0];
        float nz = (pos[3 * i + 2] - mn[2]) * inv[2];
        fixed[i] = (nz < 0.01f && (nx > 0.99f || nx < 0.01f)) ? 1 : 0;
    }
    return ATS_OK;
}

int ats_mass_area_weighted(const float* pos, int nv, const int* faces, int nf, float total, float* mass) {
    if (!pos || !faces || !mass || nv <= 0 || nf <= 0 || !(total > 0.f)) {
        set_error("ats_mass_area_weighted: bad arguments");
        return ATS_ERR_INVALID;
    }
    std::vector<double> m(nv, 0.0);
    double area = 0.0;
    for (int f = 0; f < nf; ++f) {
        int a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) {
            set_error("ats_mass_area_weighted: face index out of range");
            return ATS_ERR_INVALID;
        }
        double u[3], w[3];
        for (int k = 0; k < 3; ++k) {
            u[k] = (double)pos[3 * b + k] - pos[3 * a + k];
            w[k] = (double)pos[3 * c + k] - pos[3 * a + k];
        }
        double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        double A = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        area += A;
        m[a] += A / 3.0;
        m[b] += A / 3.0;
        m[c] += A / 3.0;
    }
    for (int i = 0; i < nv; ++i) mass[i] = (float)(m[i] / area * (double)total);
    return ATS_OK;
}

int ats_obj_read(const char* path, int* num_verts, float* positions, int* num_faces, int* faces) {
    if (!path || !num_verts || !num_faces) {
        set_error("ats_obj_read: bad arguments");
        return ATS_ERR_INVALID;
    }
    std::ifstream in(path);
    if (!in) {
        set_error(std::string("ats_obj_read: cannot open ") + path);
        return ATS_ERR_INVALID;
    }
    std::vector<float> p;
    std::vector<int> f;
    std::string line;
    while (std::getline(in, line)) {
        if (line.size() < 2) continue;
        if (line[0] == 'v' && line[1] == ' ') {
            float x, y, z;
            if (std::sscanf(line.c_str() + 2, "%f %f %f", &x, &y, &z) == 3) {
                p.push_back(x);
                p.push_back(y);
                p.push_back(z);
            }
        } else if (line[0] == 'f' && line[1] == ' ') {
            std::istringstream ss(line.substr(2));
            std::string tok;
            std::vector<int> ids;
            while (ss >> tok) {
                int idx = std::atoi(tok.c_str());
                ids.push_back(idx > 0 ? idx - 1 : (int)(p.size() / 3) + idx);
            }
            // polygons become a fan from their first vertex; degenerate triangles are dropped
            for (size_t k = 2; k < ids.size(); ++k) {
                const int a = ids[0], b = ids[k - 1], c = ids[k];
                if (a == b || a == c || b == c) continue;
                f.push_back(a);
                f.push_back(b);
                f.push_back(c);
            }
        }
    }
    int nv = (int)p.size() / 3, nf = (int)f.size() / 3;
    if (positions) {
        if (*num_verts < nv) {
            set_error("ats_obj_read: positions array too small");
            return ATS_ERR_INVALID;
        }
        std::memcpy(positions, p.data(), p.size() * sizeof(float));
    }
    if (faces) {
        if (*num_faces < nf) {
            set_error("ats_obj_read: faces array too small");
            return ATS_ERR_INVALID;
        }
        std::memcpy(faces, f.data(), f.size() * sizeof(int));
    }
    *num_verts = nv;
    *num_faces = nf;
    return ATS_OK;
}

int ats_topology_build(const ats_instance_desc* mesh, ats_topology** out) {
    if (!mesh || !out) {
        set_error("ats_topology_build: null argument");
        return ATS_ERR_INVALID;
    }
    auto* h = new (std::nothrow) ats_topology();
    if (!h) {
        set_error("ats_topology_build: out of memory");
        return ATS_ERR_NOMEM;
    }
    std::string err;
    if (!build_topology(*mesh, h->t, err)) {
        delete h;
        set_error("ats_topology_build: " + err);
        return ATS_ERR_INVALID;
    }
    *out = h;
    return ATS_OK;
}

int ats_topology_destroy(ats_topology* topo) {
    delete topo;
    return ATS_OK;
}

int ats_topology_counts(const ats_topology* topo, int* counts) {
    if (!topo || !counts) {
        set_error("ats_topology_counts: null argument");
        return ATS_ERR_INVALID;
    }
    counts[0] = topo->t.ne();
    counts[1] = topo->t.nb();
    counts[2] = topo->t.nvc();
    counts[3] = topo->t.nsc();
    counts[4] = topo->t.nbc();
    return ATS_OK;
}

int ats_topology_edges(const ats_topology* topo, int* edges, int* bending) {
    if (!topo) {
        set_error("ats_topology_edges: null topology");
        return ATS_ERR_INVALID;
    }
    if (edges) std::memcpy(edges, topo->t.edges.data(), topo->t.edges.size() * sizeof(int));
    if (bending) std::memcpy(bending, topo->t.bending.data(), topo->t.bending.size() * sizeof(int));
    return ATS_OK;
}

int ats_topology_rest(const ats_topology* topo, float* rest, float* q) {
    if (!topo) {
        set_error("ats_topology_rest: null topology");
        return ATS_ERR_INVALID;
    }
    if (rest) std::memcpy(rest, topo->t.rest.data(), topo->t.rest.size() * sizeof(float));
    if (q) std::memcpy(q, topo->t.q.data(), topo->t.q.size() * sizeof(float));
    return ATS_OK;
}

int ats_topology_coloring(const ats_topology* topo, int which, int* prefix, int* items) {
    if (!topo || !prefix || !items) {
        set_error("ats_topology_coloring: null argument");
        return ATS_ERR_INVALID;
    }
    const std::vector<int>* off;
    const std::vector<int>* it;
    switch (which) {
        case ATS_COLORING_VERTEX: off = &topo->t.vcol_off; it = &topo->t.vcol; break;
        case ATS_COLORING_STRETCH: off = &topo->t.scol_off; it = &topo->t.scol; break;
        case ATS_COLORING_BENDING: off = &topo->t.bcol_off; it = &topo->t.bcol; break;
        default: set_error("ats_topology_coloring: unknown colouring"); return ATS_ERR_INVALID;
    }
    std::memcpy(prefix, off->data(), off->size() * sizeof(int));
    std::memcpy(items, it->data(), it->size() * sizeof(int));
    return ATS_OK;
}

}  // extern "C"
