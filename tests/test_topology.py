"""Host topology of libats_b200 against the oracle (bit-exact integers and floats).

Mirrors what libAtsSim's examples print at start-up: edge / bending-edge counts
(src/Utils/mesh_reader.h:206-298) and the colour counts of
examples/example2_async_iter.cpp:458-646.
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _square8k():
    m = np.load(os.path.join(GOLD, "square8k_mesh.npz"))
    return m["positions"], m["faces"]


def _compare(ats, oracle, pos, faces):
    fixed = ats.reference_pins(pos)
    assert (fixed == oracle.reference_pins(pos)).all()
    mass = np.full(len(pos), 0.01, np.float32)
    T = ats.Topology(ats.Instance(pos, faces, mass, fixed, 1e4, 2.5e-3))
    S = oracle.Scene(pos, faces, mass, fixed)
    e, b = T.edges()
    assert np.array_equal(e, S.edges())
    assert np.array_equal(b, S.bending_edges())
    L, Q = T.rest()
    L2, Q2 = S.rest()
    assert np.array_equal(L.view(np.int32), L2.view(np.int32))
    assert np.array_equal(Q.view(np.int32), Q2.view(np.int32))
    for which in ("vertex", "stretch", "bending"):
        a, o = T.coloring(which), S.coloring(which)
        assert len(a) == len(o)
        for x, y in zip(a, o):
            assert np.array_equal(x, y)
    return T, S


def test_square8k_topology_matches_oracle(ats, oracle):
    pos, faces = _square8k()
    T, _ = _compare(ats, oracle, pos, faces)
    assert (T.ne, T.nb) == (24435, 24027)
    # colour sizes of the reference greedy vertex colouring on square8K.obj
    assert [len(c) for c in T.coloring("vertex")] == [1384, 1226, 1194, 1144, 1087, 971, 757, 430, 85, 4]


@pytest.mark.parametrize("n,pattern,ne,nb,ncol", [
    (64, 0, 12033, 11781, 4),
    (128, 0, 48641, 48133, 4),
    (64, 1, 12033, 11781, 7),
    (17, 0, 3 * 16 * 16 + 2 * 16, 3 * 16 * 16 + 2 * 16 - 4 * 16, 4),
])
def test_grid_topology(ats, oracle, n, pattern, ne, nb, ncol):
    pos, faces = ats.grid_mesh(n, pattern)
    T, _ = _compare(ats, oracle, pos, faces)
    assert (T.ne, T.nb, T.n_vcolors) == (ne, nb, ncol)
    if n == 64 and pattern == 1:
        assert [len(c) for c in T.coloring("vertex")] == [1024, 1023, 543, 497, 469, 439, 101]


def test_colorings_are_independent_sets(ats):
    pos, faces = _square8k()
    inst = ats.Instance(pos, faces, np.ones(len(pos), np.float32), np.zeros(len(pos), np.uint8), 1.0, 1.0)
    T = ats.Topology(inst)
    e, b = T.edges()
    col = np.full(len(pos), -1)
    for c, vs in enumerate(T.coloring("vertex")):
        col[vs] = c
    assert (col >= 0).all()
    # no edge and no bending-edge pair inside one colour
    assert (col[e[:, 0]] != col[e[:, 1]]).all()
    for i in range(4):
        for j in range(i + 1, 4):
            assert (col[b[:, i]] != col[b[:, j]]).all()
    for which, elems in (("stretch", e), ("bending", b)):
        for cl in T.coloring(which):
            verts = elems[cl].ravel()
            assert len(np.unique(verts)) == len(verts)


def test_alternating_grid_is_square40k_layout(ats):
    g = json.load(open(os.path.join(GOLD, "square40k_faces.json")))
    pos, faces = ats.grid_mesh(200, ats.GRID_ALTERNATING)
    assert hashlib.sha256(faces.tobytes()).hexdigest() == g["faces_sha256"]
    assert np.allclose(pos.min(0), g["bounds_min"]) and np.allclose(pos.max(0), g["bounds_max"])


def test_degenerate_faces_dropped_and_bad_index_rejected(ats):
    pos, faces = ats.grid_mesh(4)
    bad = np.concatenate([faces, [[0, 0, 1]]]).astype(np.int32)
    T = ats.Topology(ats.Instance(pos, bad, np.ones(16, np.float32), np.zeros(16, np.uint8), 1.0, 1.0))
    T0 = ats.Topology(ats.Instance(pos, faces, np.ones(16, np.float32), np.zeros(16, np.uint8), 1.0, 1.0))
    assert (T.ne, T.nb) == (T0.ne, T0.nb)
    oob = np.concatenate([faces, [[0, 1, 99]]]).astype(np.int32)
    with pytest.raises(ats.AtsError):
        ats.Topology(ats.Instance(pos, oob, np.ones(16, np.float32), np.zeros(16, np.uint8), 1.0, 1.0))


def test_single_triangle_and_isolated_vertex(ats, oracle):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1], [5, 5, 5]], np.float32)
    faces = np.array([[0, 1, 2]], np.int32)
    T, S = _compare(ats, oracle, pos, faces)
    assert (T.ne, T.nb) == (3, 0)
    assert T.n_vcolors == S.n_vcolors == 3
    assert T.n_bcolors == 1 and len(T.coloring("bending")[0]) == 0


def test_area_weighted_mass(ats):
    pos, faces = ats.grid_mesh(64)
    m = ats.mass_area_weighted(pos, faces, 0.1)
    assert abs(m.sum() - 0.1) < 1e-6
    # interior vertex of a uniform-diagonal grid touches 6 triangles of area a/2
    a = (1.0 / 63) ** 2
    assert abs(m[32 * 64 + 32] - 0.1 * 6 * (a / 2) / 3) < 1e-9


def test_obj_reader_roundtrip(ats, tmp_path):
    pos, faces = ats.grid_mesh(5, ats.GRID_ALTERNATING)
    p = tmp_path / "g.obj"
    with open(p, "w") as f:
        for v in pos:
            f.write("v %.9g %.9g %.9g\n" % tuple(v))
        for t in faces + 1:
            f.write("f %d/%d %d/%d %d/%d\n" % (t[0], t[0], t[1], t[1], t[2], t[2]))
        f.write("f 1 1 2\n")
    p2, f2 = ats.obj_read(str(p))
    assert np.array_equal(f2, faces)
    assert np.array_equal(p2, pos)
