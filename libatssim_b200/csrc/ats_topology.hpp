// ats_topology.hpp -- host-side mesh topology and colour-major device layout.
//
// Topology reproduces the reference's integer results exactly:
//   edges / bending edges      src/Utils/mesh_reader.h:206-298
//   vertex -> edge / bending CSR, vertex adjacency with bending
//                              examples/example2_async_iter.cpp:229-304
//   greedy colourings          examples/example2_async_iter.cpp:458-533 (constraints),
//                              :572-646 (vertices)
//   rest length, Q             examples/example2_async_iter.cpp:309-375
// The layout turns one or more instances into the arrays the CUDA kernels read:
// vertices ordered instance-major, colour-major inside an instance; a per-vertex
// neighbour stencil in sliced-ELL form; colour-sorted XPBD constraint arrays.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ats_cloth.h"

namespace ats {

struct Topology {
    int nv = 0, nf = 0;
    std::vector<float> pos;     // 3 nv
    std::vector<int> faces;     // 3 nf
    std::vector<int> edges;     // 2 E   (reference order: sorted (v0 < v1))
    std::vector<int> bending;   // 4 B   (v0, v1, opposite in first face, opposite in second)
    std::vector<float> rest;    // E
    std::vector<float> q;       // 16 B, column-major Q[e][col][row]
    std::vector<int> ve_off, ve;  // vertex -> adjacent edges (eid order)
    std::vector<int> vb_off, vb;  // vertex -> adjacent bending edges (eid order)
    std::vector<int> vcol_off, vcol;  // vertex colours
    std::vector<int> scol_off, scol;  // stretch colours
    std::vector<int> bcol_off, bcol;  // bending colours
    int ne() const { return (int)rest.size(); }
    int nb() const { return (int)(bending.size() / 4); }
    int nvc() const { return (int)vcol_off.size() - 1; }
    int nsc() const { return (int)scol_off.size() - 1; }
    int nbc() const { return (int)bcol_off.size() - 1; }
};

// Returns false and fills err on a malformed mesh.
bool build_topology(const ats_instance_desc& d, Topology& t, std::string& err);

// Host copy of everything the device needs, for all instances of a handle.
struct Layout {
    int tpv = 4;          // lanes per vertex in the VBD sweep
    int nv = 0, ne = 0, nb = 0, ninst = 0;
    int n_vcolors = 0, n_scolors = 0, n_bcolors = 0;
    std::vector<int> inst_vbegin;   // ninst + 1, in layout order (= caller order offsets)
    std::vector<int> to_layout;     // caller vertex id -> layout id
    std::vector<int> to_caller;     // layout id -> caller vertex id
    // per-vertex, layout order (float4 as 4 floats)
    std::vector<float> x0;          // xyz rest position, w = mass
    std::vector<float> vel;         // zeros
    std::vector<float> vm;          // {bending Hessian diagonal k_b sum Q_oo, pin boost (0 / 1e9), inv mass, instance id bits}
    std::vector<float> inst;        // per instance {gravity xyz, k_stretch}
    // neighbour lists (CSR, layout order): neighbour id, rest length (-1 = not an
    // edge), bending weight k_b sum_b Q_b[o_v][o_u]; per vertex the edge neighbours
    // come first (nb_nedge of them), then the bending-only ones, each group sorted by id
    std::vector<int> nb_off, nb_u, nb_nedge;
    std::vector<float> nb_rest, nb_w;
    std::vector<int> runs;          // per colour c: runs[c] .. runs of (begin, end) layout ranges
    std::vector<int> run_off;       // n_vcolors + 1 offsets into runs (pairs)
    // sliced-ELL stencil for the current tpv: slice = 32/tpv vertices, row r holds 32
    // entries; the first edge rows hold edge neighbours, the remaining rows the
    // bending-only neighbours (far corners of bending edges)
    std::vector<int> st_iw;         // 2 per entry: neighbour layout id (self for padding), bending weight bits
    std::vector<float> st_rest;     // per entry: rest length (edge rows only), -1 = padding
    std::vector<int> slices;        // 4 ints per slice: vbegin, nverts, entry offset, rows | edge rows << 16
    std::vector<int> color_slices;  // n_vcolors + 1 offsets into slices
    // XPBD, colour-major over all instances
    std::vector<int> xs_edge;       // 2 per constraint (layout ids)
    std::vector<float> xs_rest, xs_k;
    std::vector<int> xs_color;      // n_scolors + 1
    std::vector<int> xb_idx;        // 4 per constraint
    std::vector<float> xb_q;        // 12 per constraint: Q00 Q01 Q02 Q03 Q11 Q12 Q13 Q22 Q23 Q33 k_b 0
    std::vector<int> xb_color;      // n_bcolors + 1
    // FP64 energy: original edges / bending edges in layout ids
    std::vector<int> en_edge;       // 2 per edge
    std::vector<float> en_rest, en_k;
    std::vector<int> en_bend;       // 4 per bending edge
    std::vector<float> en_q;        // 16 per bending edge (column-major)
    std::vector<float> en_kb;
    std::vector<int> inst_eseg, inst_bseg;  // ninst + 1 offsets into en_edge / en_bend pairs
    // learned warm start: per vertex the edge neighbours in 6 rest-direction slots
    // (+x, +x+z, +z, -x, -x-z, -z in the rest plane; -1 = none) and their rest lengths
    std::vector<int> feat_nb;       // 6 per vertex, layout ids
    std::vector<float> feat_len;    // 6 per vertex
};

bool build_layout(const std::vector<Topology>& topos, const std::vector<ats_instance_desc>& descs, const float* gravity,
                  int tpv, Layout& L, std::string& err);
// (Re)builds the sliced-ELL stencil of L for `tpv` lanes per vertex.
bool build_slices(Layout& L, int tpv, std::string& err);

}  // namespace ats
