"""Oracle parity on every configuration the benchmark times, through the C ABI.

Each test runs the CUDA solver and the CPU oracle (a restatement of the reference's
CPU VBD / XPBD, examples/example2_async_iter.cpp:1017-1143 with the terms of
src/Solver/xpbd_constraints.h) on the same scene, the same colourings and the same
iteration count, frame by frame, and compares positions.

Bars (relative L2 of positions, FP32):
  VBD   1e-4  the CUDA sweep sums the merged per-neighbour bending weights in its own
              order, so roundings differ from the oracle's;
  XPBD  1e-5  every term is rounded explicitly in the reference's order (the c0 test
              of test_vbd_gpu.py holds it to 1e-6; at 512^2 x 50 iterations x 30 frames
              the bar leaves room for the sqrt / division roundings to drift).
"""
import os

import numpy as np
import pytest

from libatssim_b200 import configs

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def scene(oracle, inst, prm, iterations=None):
    return oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, dt=prm["implicit_dt"],
                        substeps=prm["num_substep"], iterations=iterations or prm["iterations"],
                        k_stretch=inst.k_stretch, k_bend=inst.k_bend, damping=prm["damping"], threads=THREADS)


def moved(x, rest):
    return float(np.linalg.norm(x - rest) / np.linalg.norm(rest))


def test_c1_vbd_thirty_frames(ats, oracle):
    """c1: 512 x 512 cloth, 50 VBD iterations per frame, 30 CUDA-graph frames."""
    insts, prm = configs.c1()
    cloth = ats.Cloth(insts, **prm)
    s = scene(oracle, insts[0], prm)
    for _ in range(30):
        cloth.frame(graph=True)
    s.run(30)
    xg, vg = cloth.state()
    xo, vo = s.state()
    assert moved(xo, insts[0].positions) > 0.05
    err = rel_l2(xg, xo)
    assert err < 1e-4, err
    assert rel_l2(vg, vo) < 1e-2
    cloth.close()


def test_c1_xpbd_thirty_frames(ats, oracle):
    """c1 solved by XPBD: 50 iterations of (stretch colours + bending colours)."""
    insts, prm = configs.c1()
    cloth = ats.Cloth(insts, **prm)
    s = scene(oracle, insts[0], prm)
    for _ in range(30):
        cloth.frame(ats.SOLVER_XPBD, graph=True)
    s.run(30, solver="xpbd")
    xg, _ = cloth.state()
    xo, _ = s.state()
    assert moved(xo, insts[0].positions) > 0.05
    err = rel_l2(xg, xo)
    assert err < 1e-5, err
    cloth.close()


def test_c0_xpbd_hundred_iterations(ats, oracle):
    """c0 at its own iteration count (100) under XPBD, 30 frames."""
    insts, prm = configs.c0()
    cloth = ats.Cloth(insts, **prm)
    s = scene(oracle, insts[0], prm)
    for _ in range(30):
        cloth.frame(ats.SOLVER_XPBD, graph=True)
    s.run(30, solver="xpbd")
    xg, _ = cloth.state()
    xo, _ = s.state()
    err = rel_l2(xg, xo)
    assert err < 1e-5, err
    cloth.close()


def c2_extremes():
    """The c2 instances at the ends of its material ranges: stiffest and softest
    springs, stiffest and softest bending (k in [1e2, 1e4] N/m, k_b in [1e-3, 1e-1])."""
    insts, prm = configs.c2()
    ks = np.array([i.k_stretch for i in insts])
    kbs = np.array([i.k_bend for i in insts])
    pick = []
    for idx in (int(np.argmax(ks)), int(np.argmin(ks)), int(np.argmax(kbs)), int(np.argmin(kbs))):
        if idx not in pick:
            pick.append(idx)
    return [insts[i] for i in pick], prm, pick


def test_c2_stiffness_extremes_batched(ats, oracle):
    """The extreme c2 instances in one batched handle, each against its own oracle
    scene (30 frames x 50 iterations)."""
    sel, prm, pick = c2_extremes()
    ks = [i.k_stretch for i in sel]
    kbs = [i.k_bend for i in sel]
    assert max(ks) > 8e3 and min(ks) < 1.3e2 and max(kbs) > 8e-2 and min(kbs) < 1.3e-3, (ks, kbs)
    cloth = ats.Cloth(sel, **prm)
    for _ in range(30):
        cloth.frame(graph=True)
    xg, _ = cloth.state()
    off = 0
    for inst in sel:
        s = scene(oracle, inst, prm)
        s.run(30)
        xo, _ = s.state()
        n = inst.num_verts
        err = rel_l2(xg[off:off + n], xo)
        assert err < 1e-4, (inst.k_stretch, inst.k_bend, err)
        off += n
    cloth.close()


def test_wind_per_frame_c3_cloth(ats, oracle):
    """c3: 128 x 128 cloth, 200 iterations, a random wind force each frame (gravity
    plus F / M on every free vertex), 30 frames; the oracle takes the same
    acceleration each frame."""
    insts, prm = configs.c3()
    inst = insts[0]
    cloth = ats.Cloth(insts, **prm)
    s = scene(oracle, inst, prm)
    total = float(inst.mass.sum())
    for f in range(30):
        a = configs.wind_accel(np.random.RandomState(10000 + f), total).astype(np.float32)
        cloth.set_accel(a[None, :])
        s.set_gravity(a)
        cloth.frame(graph=True)
        s.frame()
    xg, _ = cloth.state()
    xo, _ = s.state()
    err = rel_l2(xg, xo)
    assert err < 1e-4, err
    cloth.close()


def test_wind_per_instance_batched(ats, oracle):
    """c4-style: batched instances of uneven side, each with its own wind per frame."""
    sides = [64, 83, 101]
    insts = [configs.grid_instance(n) for n in sides]
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=50, damping=2.0)
    cloth = ats.Cloth(insts, **prm)
    scenes = [scene(oracle, i, prm) for i in insts]
    masses = [float(i.mass.sum()) for i in insts]
    for f in range(20):
        acc = np.stack([configs.wind_accel(np.random.RandomState(777 + 31 * f + k), m)
                        for k, m in enumerate(masses)]).astype(np.float32)
        cloth.set_accel(acc)
        cloth.frame(graph=True)
        for k, sc in enumerate(scenes):
            sc.set_gravity(acc[k])
            sc.frame()
    xg, _ = cloth.state()
    off = 0
    for inst, sc in zip(insts, scenes):
        xo, _ = sc.state()
        n = inst.num_verts
        err = rel_l2(xg[off:off + n], xo)
        assert err < 1e-4, (inst.num_verts, err)
        off += n
    cloth.close()


@pytest.mark.parametrize("policy", [0, 1])
def test_frame_to_residual_matches_oracle(ats, oracle, policy):
    """The residual-driven frame: the same stopping iteration as the oracle's
    to-residual frame (probes every 5 iterations, or the extrapolated schedule) and the
    same positions."""
    inst = configs.grid_instance(48)
    prm = dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=50, damping=2.0)
    cloth = ats.Cloth([inst], **prm)
    cloth.set_probe_policy(policy)
    s = scene(oracle, inst, prm)
    agree = 0
    for f in range(12):
        it_g, r_g = cloth.frame_to_residual(0.3, check_every=5, max_iterations=200)
        it_o, r_o = s.frame_to_residual(0.3, check_every=5, max_iterations=200, policy=policy)
        # the probes sum FP32 force terms in FP64, the oracle is FP64 throughout: near
        # the threshold they may stop one probe apart
        assert abs(int(it_g[0]) - it_o) <= 5, (f, it_g, it_o)
        assert abs(r_g[0] - r_o) < 2e-3 * max(1.0, r_o) or it_g[0] != it_o, (f, r_g, r_o)
        agree += int(it_g[0]) == it_o
        if int(it_g[0]) != it_o:  # resynchronise the two trajectories
            x, v = s.state()
            cloth.set_state(x, v)
    assert agree >= 10
    xg, _ = cloth.state()
    xo, _ = s.state()
    assert rel_l2(xg, xo) < 1e-4
    cloth.close()
