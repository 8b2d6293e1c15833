"""CUDA VBD / XPBD against the CPU oracle, through the C ABI.

Bars: positions within 1e-4 relative L2 after 30 frames in FP32 (FP32 summation
order differs: the CUDA sweep merges bending terms per neighbour); FP64 energies
and residuals within 1e-6 relative of the oracle's on the same positions.
"""
import json
import os

import numpy as np
import pytest

from libatssim_b200 import configs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_scene(oracle, inst, prm, threads=4):
    return oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, dt=prm["implicit_dt"],
                        substeps=prm["num_substep"], iterations=prm["iterations"], k_stretch=inst.k_stretch,
                        k_bend=inst.k_bend, damping=prm["damping"], threads=threads)


def perturbed_state(inst, seed, vscale=0.3, xscale=1e-3):
    rng = np.random.RandomState(seed)
    x = inst.positions + xscale * rng.standard_normal(inst.positions.shape).astype(np.float32)
    v = vscale * rng.standard_normal(inst.positions.shape).astype(np.float32)
    return x.astype(np.float32), v


@pytest.mark.parametrize("tpv", [1, 2, 4, 8])
def test_one_frame_matches_oracle(ats, oracle, tpv):
    insts, prm = configs.c0()
    prm = dict(prm, iterations=3)
    inst = insts[0]
    x, v = perturbed_state(inst, seed=tpv)
    cloth = ats.Cloth(insts, threads_per_vertex=tpv, **prm)
    cloth.set_state(x, v)
    cloth.frame()
    xg, vg = cloth.state()
    s = oracle_scene(oracle, inst, prm)
    s.set_state(x, v)
    s.frame()
    xo, vo = s.state()
    assert rel_l2(xg, xo) < 1e-6
    assert rel_l2(vg - v, vo - v) < 1e-4


def test_c0_thirty_frames_vbd(ats, oracle):
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    s = oracle_scene(oracle, insts[0], prm, threads=8)
    for _ in range(30):
        cloth.frame(graph=True)
    s.run(30)
    xg, vg = cloth.state()
    xo, vo = s.state()
    rest = insts[0].positions
    err = rel_l2(xg, xo)
    assert err < 1e-4, err
    # the cloth has fallen well away from rest: the comparison is not trivial
    assert np.linalg.norm(xo - rest) / np.linalg.norm(rest) > 0.05
    assert rel_l2(xg - rest, xo - rest) < 1e-3


def test_c0_thirty_frames_xpbd(ats, oracle):
    insts, prm = configs.c0()
    prm = dict(prm, iterations=20)
    cloth = ats.Cloth(insts, **prm)
    s = oracle_scene(oracle, insts[0], prm, threads=8)
    for _ in range(30):
        cloth.frame(ats.SOLVER_XPBD)
    s.run(30, solver="xpbd")
    xg, _ = cloth.state()
    xo, _ = s.state()
    # predict / update / XPBD kernels round every term as the oracle does
    assert rel_l2(xg, xo) < 1e-6


def test_square8k_energy_log_matches_reference(ats, oracle):
    """GPU reproduction of documents/example2_async_convergence.py:78-80."""
    m = np.load(os.path.join(GOLD, "square8k_mesh.npz"))
    insts, prm = configs.reference_square(m["positions"], m["faces"])
    cloth = ats.Cloth(insts, **prm)
    for _ in range(30):
        cloth.frame(graph=True)
    gold = np.array(json.load(open(os.path.join(GOLD, "example2_energy_frame30.json")))["list_sync"])
    cloth.predict()
    log = [cloth.energy()[:2].sum()]
    for _ in range(100):
        for c in range(cloth.info.num_vertex_colors):
            cloth.vbd_color_sweep(c)
        log.append(cloth.energy()[:2].sum())
    cloth.update_velocity()
    log = np.array(log)
    assert np.max(np.abs(log - gold) / gold) < 2e-5
    assert (np.diff(log) < 0).all()


def test_energy_and_residual_match_oracle(ats, oracle):
    insts, prm = configs.c0()
    inst = insts[0]
    x, v = perturbed_state(inst, seed=7, vscale=0.1)
    cloth = ats.Cloth(insts, **prm)
    cloth.set_state(x, v)
    cloth.predict()
    for c in range(cloth.info.num_vertex_colors):
        cloth.vbd_color_sweep(c)
    xm = cloth.positions()
    s = oracle_scene(oracle, inst, prm)
    s.set_state(x, v)
    s.begin_frame()
    e = cloth.energy()
    eo = s.energy_of(xm, with_bending=False)
    assert abs(e[0] + e[1] - eo) / eo < 1e-6
    r = cloth.residual()[0]
    ro = s.grad_norm_of(xm)
    assert abs(r - ro) / ro < 1e-6


def test_graph_replay_is_bit_identical_to_eager(ats):
    insts, prm = configs.c0()
    a = ats.Cloth(insts, **prm)
    b = ats.Cloth(insts, **prm)
    for _ in range(3):
        a.frame()
        b.frame(graph=True)
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    b.close()  # gives back the persisting-L2 set-aside


def test_lane_variants_agree(ats):
    insts, prm = configs.c0()
    out = []
    for tpv in (1, 2, 4, 8):
        c = ats.Cloth(insts, threads_per_vertex=tpv, **prm)
        for _ in range(5):
            c.frame(graph=True)
        out.append(c.state()[0])
    for o in out[1:]:
        assert rel_l2(o, out[0]) < 1e-5


def test_autotune_keeps_state_and_parity(ats, oracle):
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    cloth.frame()
    x_before = cloth.positions()
    tpv, block = cloth.autotune(iterations=2)
    assert tpv in (1, 2, 4, 8) and block in (64, 128, 256)
    assert cloth.info.threads_per_vertex == tpv and cloth.info.block_size == block
    assert np.array_equal(cloth.positions(), x_before)
    for _ in range(9):
        cloth.frame(graph=True)
    s = oracle_scene(oracle, insts[0], prm, threads=8)
    s.run(10)
    assert rel_l2(cloth.state()[0], s.state()[0]) < 1e-4


def test_batched_instances_equal_separate_handles(ats):
    insts, prm = configs.c2(num_instances=5, seed=3, side_range=(8, 40))
    prm = dict(prm, iterations=10)
    batch = ats.Cloth(insts, **prm)
    for _ in range(3):
        batch.frame(graph=True)
    xb, vb = batch.state()
    off = 0
    for inst in insts:
        one = ats.Cloth([inst], **prm)
        for _ in range(3):
            one.frame()
        x1, v1 = one.state()
        n = inst.num_verts
        assert np.array_equal(xb[off:off + n], x1)
        assert np.array_equal(vb[off:off + n], v1)
        off += n


def test_residual_decreases_over_iterations(ats):
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    for _ in range(5):
        cloth.frame()
    cloth.predict()
    r0 = cloth.residual()[0]
    for _ in range(50):
        for c in range(cloth.info.num_vertex_colors):
            cloth.vbd_color_sweep(c)
    assert cloth.residual()[0] < 0.5 * r0


def test_pinned_vertices_stay(ats, oracle):
    """Pins are the reference's 1e9 penalty on the inertia Hessian
    (xpbd_constraints.h:4056-4060), so they move by (tension / 1e9) per iteration."""
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    s = oracle_scene(oracle, insts[0], prm, threads=8)
    for _ in range(10):
        cloth.frame(graph=True)
    s.run(10)
    x, _ = cloth.state()
    xo, _ = s.state()
    pinned = insts[0].fixed.astype(bool)
    drift = np.abs(x[pinned] - insts[0].positions[pinned]).max()
    drift_o = np.abs(xo[pinned] - insts[0].positions[pinned]).max()
    assert drift < 1e-4 and abs(drift - drift_o) < 0.05 * drift_o + 1e-9
    assert x[~pinned, 1].min() < -0.1


def test_bad_color_is_rejected(ats):
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    with pytest.raises(ats.AtsError):
        cloth.vbd_color_sweep(cloth.info.num_vertex_colors)
    with pytest.raises(ats.AtsError):
        cloth.xpbd_stretch_color(-1)


def test_frame_to_residual_matches_explicit_iterations(ats):
    insts, prm = configs.c0()
    a = ats.Cloth(insts, **prm)
    b = ats.Cloth(insts, **prm)
    for _ in range(5):
        a.frame(graph=True)
        b.frame(graph=True)
    its, res = a.frame_to_residual(tol=0.25, check_every=5, max_iterations=400)
    assert its[0] % 5 == 0 and 0 < its[0] <= 400
    assert res[0] <= 0.25 or its[0] == 400
    # the same frame by hand: predict, the same number of iterations, residual, update
    b.predict()
    r0 = b.residual()[0]
    b.vbd_iterations(int(its[0]))
    r1 = b.residual()[0]
    b.update_velocity()
    # the frame's probes use FP32 per-vertex gradient terms, ats_residual FP64 ones: a
    # spring's l - L at ~1e-3 strain and the inertia term's x - y beside x - x0 cancel,
    # leaving ~1e-4 of the residual (the solver's own forces have the same floor)
    assert abs(r1 / r0 - res[0]) <= 2e-4 * res[0]
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_batched_early_exit_per_instance(ats):
    insts, prm = configs.c2(num_instances=6, seed=5, side_range=(8, 48))
    batch = ats.Cloth(insts, **prm)
    for _ in range(2):
        batch.frame(graph=True)
    x_start, v_start = batch.state()
    its, res = batch.frame_to_residual(tol=0.05, check_every=4, max_iterations=300)
    assert len(set(its.tolist())) > 1  # instances stop at different iteration counts
    xb, vb = batch.state()
    off = 0
    for i, inst in enumerate(insts):
        n = inst.num_verts
        one = ats.Cloth([inst], **prm)
        one.set_state(x_start[off:off + n], v_start[off:off + n])
        one.predict()
        one.vbd_iterations(int(its[i]))
        one.update_velocity()
        x1, v1 = one.state()
        assert np.array_equal(xb[off:off + n], x1), i
        assert np.array_equal(vb[off:off + n], v1), i
        off += n


def _potential_fp64(ats, inst, x, x0, v0, h, accel):
    """G(x) of one instance in FP64 from its own topology: inertia against
    y = x0 + h v0 + h^2 a (a = 0 at pins), springs 1/2 k (l - L)^2, bending
    1/2 k_b sum_b x^T Q_b x."""
    topo = ats.Topology(inst)
    e, b = topo.edges()
    L, Q = topo.rest()
    x, x0, v0 = (np.asarray(a, dtype=np.float64) for a in (x, x0, v0))
    # material and acceleration as the handle stores them (FP32)
    ks, kb = float(np.float32(inst.k_stretch)), float(np.float32(inst.k_bend))
    acc = np.asarray(accel, dtype=np.float32).astype(np.float64)
    a = np.where(inst.fixed[:, None] != 0, 0.0, acc[None, :])
    d = x - (x0 + h * v0 + h * h * a)
    gi = np.sum(inst.mass.astype(np.float64) / (2 * h * h) * np.sum(d * d, axis=1))
    l = np.linalg.norm(x[e[:, 1]] - x[e[:, 0]], axis=1)
    gs = np.sum(0.5 * ks * (l - L.astype(np.float64)) ** 2)
    P = x[b]  # (B, 4, 3)
    Qd = Q.astype(np.float64)
    gb = 0.5 * kb * np.einsum("bij,bik,bjk->", Qd, P, P)
    # size of the terms the per-vertex form adds: sum |k_b Q_ij| |x_i - x_j|^2
    D = np.sum((P[:, :, None, :] - P[:, None, :, :]) ** 2, axis=3)
    scale = kb * np.sum(np.abs(Qd) * D)
    return gi + gs + gb, scale


@pytest.mark.parametrize("bending", [True, False])
def test_potential_matches_fp64_evaluation(ats, bending):
    insts, prm = configs.c2(num_instances=3, seed=5, side_range=(10, 24))
    if not bending:
        insts = [ats.Instance(i.positions, i.faces, i.mass, i.fixed, i.k_stretch, 0.0) for i in insts]
    cloth = ats.Cloth(insts, **prm)
    for _ in range(3):
        cloth.frame()
    x0, v0 = cloth.state()
    cloth.predict()
    cloth.vbd_iterations(7)
    x = cloth.positions()
    cloth.set_state(x0, v0)
    cloth.set_positions(x)
    g = cloth.potential()
    h = float(np.float32(prm["implicit_dt"]))  # the handle keeps h in FP32
    o = 0
    for i, inst in enumerate(insts):
        n = inst.num_verts
        ref, scale = _potential_fp64(ats, inst, x[o:o + n], x0[o:o + n], v0[o:o + n], h, (0.0, -9.8, 0.0))
        # the kernel sums -1/4 W_vu |x_u - x_v|^2 with the solver's merged weights W,
        # FP32 sums of k_b Q (~1e-7 relative rounding per term, random in sign); the
        # terms are large and cancel, so the bending part carries ~1e-9 of their size
        assert abs(g[i] - ref) <= 5e-9 * scale + 1e-9 * abs(ref), (i, g[i], ref, scale)
        o += n


def test_scheduled_probes_stop_at_first_due_point(ats):
    # probes do not change the iterate, so an instance probed on a schedule stops at
    # the first point of its schedule at or after the count a probe-every-iteration
    # run finds (or at the cap)
    insts, prm = configs.c2(num_instances=6, seed=11, side_range=(12, 40))
    a = ats.Cloth(insts, **prm)
    for _ in range(2):
        a.frame()
    x0, v0 = a.state()
    tols = np.full(len(insts), 0.2)
    need, _ = a.frame_to_residual(tols, check_every=1, max_iterations=120)
    first = np.array([3, 7, 1, 20, 11, 5], dtype=np.int32)
    step = 4
    a.set_state(x0, v0)
    got, res = a.frame_to_residual(tols, check_every=step, max_iterations=120, first_check=first)
    for i in range(len(insts)):
        pts = [k for k in range(first[i], 121, step)] + [120]
        expect = min(p for p in pts if p >= need[i])
        assert got[i] == expect, (i, need[i], got[i], expect)
        assert res[i] <= 0.2 or got[i] == 120


def test_frame_probe_residual_matches_fp64_residual(ats):
    # the residual-driven frame probes with FP32 per-vertex gradient terms (FP64 sums);
    # its reported residual agrees with the FP64 ats_residual of the same iterate to
    # the FP32 cancellation floor of those terms (~1e-4 of the residual)
    insts, prm = configs.c2(num_instances=3, seed=4, side_range=(16, 30))
    cloth = ats.Cloth(insts, **prm)
    for _ in range(2):
        cloth.frame()
    x0, v0 = cloth.state()
    its, r_frame = cloth.frame_to_residual(np.zeros(len(insts)), check_every=6, max_iterations=6)
    assert (its == 6).all()
    cloth.set_state(x0, v0)
    cloth.predict()
    n_y = cloth.residual()
    cloth.vbd_iterations(6)
    r64 = cloth.residual() / n_y
    assert np.allclose(r_frame, r64, rtol=2e-4, atol=0), (r_frame, r64)


def _fan_instance(ats, k=40):
    """A fan of k triangles around one vertex: the centre has k edge neighbours, far
    more stencil rows than the sweep loads up front."""
    t = np.linspace(0.0, 2 * np.pi, k, endpoint=False)
    pos = np.concatenate([[[0.0, 0.0, 0.0]], np.stack([0.3 * np.cos(t), 0.02 * np.sin(3 * t), 0.3 * np.sin(t)], 1)])
    pos = pos.astype(np.float32)
    faces = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], dtype=np.int32)
    fixed = np.zeros(k + 1, dtype=np.uint8)
    fixed[[1, 1 + k // 2]] = 1
    mass = ats.mass_area_weighted(pos, faces, 0.05)
    return ats.Instance(pos, faces, mass, fixed, 500.0, 5e-3)


def _ragged_instance(ats):
    """An 8 x 8 grid with a third face on one interior edge (non-manifold), an
    isolated vertex and a detached triangle."""
    pos, faces = ats.grid_mesh(8)
    nv = pos.shape[0]
    a, b = 3 * 8 + 3, 3 * 8 + 4  # an interior edge of the grid
    flap = (pos[a] + pos[b]) / 2 + np.array([0.0, 0.08, 0.0], dtype=np.float32)
    extra = np.array([flap, [0.5, 0.3, 0.5], [1.3, 0.0, 0.0], [1.4, 0.0, 0.0], [1.3, 0.0, 0.1]], dtype=np.float32)
    pos = np.concatenate([pos, extra]).astype(np.float32)
    faces = np.concatenate([faces, [[a, b, nv], [nv + 2, nv + 3, nv + 4]]]).astype(np.int32)
    fixed = np.zeros(pos.shape[0], dtype=np.uint8)
    fixed[[0, 7]] = 1
    mass = ats.mass_area_weighted(pos, faces, 0.1)
    return ats.Instance(pos, faces, mass, fixed, 1e3, 1e-2)


@pytest.mark.parametrize("mesh", ["fan", "ragged"])
def test_irregular_meshes_match_oracle(ats, oracle, mesh):
    inst = _fan_instance(ats) if mesh == "fan" else _ragged_instance(ats)
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=30, damping=2.0)
    s = oracle_scene(oracle, inst, prm)
    s.run(10)
    xo, _ = s.state()
    for tpv in (1, 8):
        cloth = ats.Cloth([inst], threads_per_vertex=tpv, **prm)
        for _ in range(10):
            cloth.frame()
        xg, _ = cloth.state()
        assert np.isfinite(xg).all()
        assert rel_l2(xg, xo) < 1e-4, (mesh, tpv, rel_l2(xg, xo))
    # XPBD rounds every term as the oracle does
    sx = oracle_scene(oracle, inst, prm)
    sx.run(10, solver="xpbd")
    cx = ats.Cloth([inst], **prm)
    for _ in range(10):
        cx.frame(ats.SOLVER_XPBD)
    assert rel_l2(cx.state()[0], sx.state()[0]) < 1e-6


@pytest.mark.parametrize("n", [32, 200])
def test_xpbd_persistent_frame_equals_per_colour_launches(ats, n):
    """XPBD frames run their iterations as one cooperative launch (every colour a
    grid-stride loop, colours separated by a grid barrier); the per-colour entry points
    launch one kernel per colour. Both evaluate the same constraint bodies in the same
    colour order, so the positions are bit-identical."""
    inst = configs.grid_instance(n)
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=12, damping=2.0)
    a = ats.Cloth([inst], **prm)
    b = ats.Cloth([inst], **prm)
    a.set_sweep_form(1, ats.SOLVER_XPBD)
    assert a.info.xpbd_form == 1
    for f in range(4):
        a.frame(ats.SOLVER_XPBD, graph=(f % 2 == 1))
        b.predict()
        b.xpbd_reset()
        for _ in range(prm["iterations"]):
            for c in range(b.info.num_stretch_colors):
                b.xpbd_stretch_color(c)
            for c in range(b.info.num_bending_colors):
                b.xpbd_bending_color(c)
        b.update_velocity()
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert np.linalg.norm(xa - inst.positions) > 1e-3


@pytest.mark.parametrize("n", [32, 256])
def test_persistent_vbd_frames_equal_per_colour_launches(ats, n):
    """Fixed-iteration VBD frames in the persistent form (all iterations in one
    cooperative launch, a grid barrier between colours) and in the one-launch-per-
    colour form evaluate the same per-vertex arithmetic in the same colour order:
    bit-identical positions, eager and as CUDA graphs."""
    inst = configs.grid_instance(n)
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=15, damping=2.0)
    a = ats.Cloth([inst], **prm)
    b = ats.Cloth([inst], **prm)
    a.set_sweep_form(1)
    b.set_sweep_form(0)
    assert a.info.vbd_form == 1 and b.info.vbd_form == 0
    for f in range(4):
        a.frame(graph=(f % 2 == 1))
        b.frame(graph=(f % 2 == 1))
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert np.linalg.norm(xa - inst.positions) > 1e-3
    a.vbd_iterations(3)
    b.vbd_iterations(3)
    assert np.array_equal(a.positions(), b.positions())


@pytest.mark.parametrize("tpv", [1, 2, 4, 8])
@pytest.mark.parametrize("form", [1, 2])
def test_list_sweep_forms_equal_plain(ats, tpv, form):
    """The residual-driven frames' sweep, plain against pipelined (each warp stages its
    next slice in shared memory while computing the current one), streamed (evict-first
    loads, next descriptor in flight, material from the slice metadata and vel.w), the
    last also with the positions persisting in L2: the same slices and the same arithmetic, so bit-identical
    positions; with some instances stopping early, pinned corners, and a state set from
    the host halfway (which must keep vel.w)."""
    insts, prm = configs.c2(num_instances=5, seed=3, side_range=(20, 90))
    a = ats.Cloth(insts, threads_per_vertex=tpv, block_size=128, **prm)
    b = ats.Cloth(insts, threads_per_vertex=tpv, block_size=128, **prm)
    a.set_list_sweep(0)
    b.set_list_sweep(form)
    if form == 2:
        b.set_l2_persisting(1)
        assert b.info.l2_persisting == 1
    assert a.info.list_form == 0 and b.info.list_form == form
    for f in range(4):
        if f == 2:
            xs, vs = a.state()
            a.set_state(xs, vs)
            b.set_state(xs, vs)
        tol = 0.0 if f % 2 == 0 else 0.35
        ia, ra = a.frame_to_residual(tol, check_every=5, max_iterations=15)
        ib, rb = b.frame_to_residual(tol, check_every=5, max_iterations=15)
        assert np.array_equal(ia, ib) and np.array_equal(ra, rb)
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_autotune_cache_hits_for_the_same_mesh_class(ats):
    """A second handle of the same GPU and mesh class takes the first one's choices from
    the autotuning cache without timing; the choices survive a save and load."""
    import os
    import tempfile
    ats.autotune_cache_clear()
    insts, prm = configs.c2(num_instances=3, seed=5, side_range=(30, 60))
    a = ats.Cloth(insts, **prm)
    shape_a = a.autotune(iterations=5)
    assert a.info.tune_source == 1 and ats.autotune_cache_size() == 1
    b = ats.Cloth(insts, **prm)
    assert b.info.tune_source == 0
    assert b.autotune(iterations=5) == shape_a
    assert b.info.tune_source == 2
    for f in ("vbd_form", "list_form", "xpbd_form"):
        assert getattr(b.info, f) == getattr(a.info, f), f
    # a different mesh class is timed
    c = ats.Cloth([configs.grid_instance(200)], **prm)
    c.autotune(iterations=5)
    assert c.info.tune_source == 1 and ats.autotune_cache_size() == 2
    # the cache through a file
    path = os.path.join(tempfile.mkdtemp(), "tune.txt")
    ats.autotune_cache_save(path)
    ats.autotune_cache_clear()
    ats.autotune_cache_load(path)
    d = ats.Cloth(insts, **prm)
    assert d.autotune(iterations=5) == shape_a and d.info.tune_source == 2
    # the same shape and forms give the same frames
    d.set_state(*a.state())
    for _ in range(2):
        a.frame()
        d.frame()
    assert np.array_equal(a.positions(), d.positions())
    for h in (a, b, c, d):
        h.close()
    ats.autotune_cache_clear()


def test_list_sweep_and_l2_switch_arguments(ats):
    """ats_set_list_sweep and ats_set_l2_persisting reject out-of-range arguments; the
    context's persisting-L2 set-aside is sized while handles hold it and put back to
    what it was when the last one lets go."""
    import cuda.bindings.runtime as rt

    def setaside():
        err, v = rt.cudaDeviceGetLimit(rt.cudaLimit.cudaLimitPersistingL2CacheSize)
        assert err == rt.cudaError_t.cudaSuccess
        return v

    insts, prm = configs.c2(num_instances=2, seed=1, side_range=(20, 30))
    a = ats.Cloth(insts, **prm)
    for bad in (-1, 3):
        with pytest.raises(ats.AtsError) as e:
            a.set_list_sweep(bad)
        assert e.value.status == ats.ATS_ERR_INVALID
    assert ats.lib().ats_set_l2_persisting(a.h, 2) == ats.ATS_ERR_INVALID
    before = setaside()
    a.set_l2_persisting(1)
    b = ats.Cloth(insts, **prm)
    b.set_l2_persisting(1)
    assert a.info.l2_persisting == 1 and b.info.l2_persisting == 1
    assert setaside() >= before
    a.set_l2_persisting(0)
    assert a.info.l2_persisting == 0
    b.close()  # the last holder
    assert setaside() == before
    a.close()


def test_edge_cases_tiny_pinned_and_empty(ats, oracle):
    """Degenerate inputs the sweeps must carry: no instances (rejected), a single triangle
    (3 vertices, no bending edge, a one-vertex slice per colour) batched with a normal
    cloth, an instance with every vertex pinned (inactive from the start of a
    residual-driven frame) and a frame with no iterations."""
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=8, damping=2.0)
    with pytest.raises(ats.AtsError) as e:
        ats.Cloth([], **prm)
    assert e.value.status == ats.ATS_ERR_INVALID
    tri_pos = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.0, 0.0, 0.1]], dtype=np.float32)
    tri = ats.Instance(tri_pos, np.array([[0, 1, 2]], dtype=np.int32), np.full(3, 0.01, np.float32),
                       np.array([1, 0, 0], dtype=np.uint8), 1e3, 1e-2)
    grid = configs.grid_instance(12)
    pinned = configs.grid_instance(6)
    pinned = ats.Instance(pinned.positions, pinned.faces, pinned.mass, np.ones(pinned.num_verts, np.uint8),
                          pinned.k_stretch, pinned.k_bend)
    cloth = ats.Cloth([tri, grid, pinned], **prm)
    x_start = cloth.state()[0].copy()
    for _ in range(3):
        cloth.frame()
    x, _ = cloth.state()
    # the triangle and the grid against their own oracle scenes
    n0, n1 = tri.num_verts, grid.num_verts
    for inst, lo in ((tri, 0), (grid, n0)):
        s = oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, iterations=8, k_stretch=inst.k_stretch,
                         k_bend=inst.k_bend)
        s.run(3)
        xo, _ = s.state()
        assert np.abs(x[lo:lo + inst.num_verts] - xo).max() <= 1e-5 * max(1.0, np.abs(xo).max())
    # pinned vertices stay put up to their 1e9 Hessian boost: gravity over 1e9 moves them
    # by about 1e-11 (the reference's compute_inertia does the same)
    assert np.abs(x[n0 + n1:] - x_start[n0 + n1:]).max() < 1e-8
    # residual-driven: the all-pinned instance runs no iteration; a zero cap runs none at all
    for form in (0, 2):
        cloth.set_list_sweep(form)
        it, res = cloth.frame_to_residual(1e-4, check_every=4, max_iterations=12)
        assert it[2] == 0 and it[1] == 12 and np.isfinite(res).all()
        it, res = cloth.frame_to_residual(1e-4, check_every=4, max_iterations=0)
        assert (it == 0).all()
    cloth.close()


def test_bounded_waits_expire_and_report(ats):
    """The device waits are bounded: a grid-barrier wait for arrivals that never come and
    an mbarrier wait on which nothing arrives both give up after their poll limit and
    report it, and the context keeps running kernels (a frame afterwards)."""
    b, m = ats.selftest_bounded_waits(4096)
    assert b == ats.ATS_ERR_TIMEOUT and m == ats.ATS_ERR_TIMEOUT
    insts, prm = configs.c2(num_instances=2, seed=2, side_range=(16, 24))
    cloth = ats.Cloth(insts, **prm)
    cloth.frame()
    assert np.isfinite(cloth.state()[0]).all()
    cloth.close()
