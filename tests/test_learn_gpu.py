"""Learned warm start: tensor-core MLP kernels against the FP64 oracle, the
recorded features against their definition, training, the potential-based
fallback, and the gain over the inertial guess."""
import numpy as np
import pytest

from libatssim_b200 import configs
from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _norm_vector(rng):
    n = np.zeros(54, dtype=np.float32)
    n[:24] = rng.uniform(-1, 1, 24)
    n[24:48] = rng.uniform(0.5, 2.0, 24)
    n[48:51] = rng.uniform(-0.1, 0.1, 3)
    n[51:54] = rng.uniform(0.05, 0.2, 3)
    return n


def test_forward_matches_oracle(ats):
    rng = np.random.RandomState(0)
    m = ats.MLP(seed=3)
    norm = _norm_vector(rng)
    m.set_normalization(norm)
    theta = m.params().astype(np.float64)
    x = rng.standard_normal((203, 24)).astype(np.float32)
    y = m.infer(x)
    yo, _, _ = MO.forward(theta, MO.normalize_inputs(x, norm))
    yo = MO.denormalize_outputs(yo, norm)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 1e-5


def test_gradient_matches_oracle(ats):
    rng = np.random.RandomState(1)
    m = ats.MLP(seed=4)
    theta = m.params().astype(np.float64)
    x = rng.standard_normal((200, 24)).astype(np.float32)  # 200 = 3 full tiles + a ragged one
    t = rng.standard_normal((200, 3)).astype(np.float32)
    loss, g = m.gradient(x, t)
    lo, go = MO.loss_and_grad(theta, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lo) / lo < 1e-5
    # FP32 accumulation vs FP64, and the odd BF16 rounding of an activation decided
    # differently from an FP32 instead of an FP64 pre-activation (~0.4 % of one element)
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 1e-3
    # every layer, weights and biases
    for a, b in ((0, 1536), (1536, 1600), (1600, 5696), (5696, 5760), (5760, 9856), (9856, 9920), (9920, 10112),
                 (10112, 10115)):
        assert np.linalg.norm(g[a:b] - go[a:b]) <= 5e-3 * np.linalg.norm(go[a:b]) + 1e-9


def test_recorded_samples_follow_definition(ats):
    inst = configs.grid_instance(12)
    cloth = ats.Cloth([inst], implicit_dt=1.0 / 60.0, num_substep=1, iterations=20, damping=2.0)
    for _ in range(3):
        cloth.frame()
    x0, v0 = cloth.state()
    ds = ats.Dataset(1000)
    cloth.predict()
    y = cloth.positions()
    cloth.record_begin()
    cloth.vbd_iterations(20)
    xs = cloth.positions()
    cloth.record_end(ds)
    f, t = ds.read()
    free = np.nonzero(inst.fixed == 0)[0]
    assert len(ds) == len(free)
    order = cloth.vertex_order()
    caller_of_layout = np.argsort(order)
    rows = caller_of_layout[np.sort(order[free])]  # free vertices in device order
    h = 1.0 / 60.0
    s = 9.8 * h * h
    assert np.allclose(f[:, 0:3], h * v0[rows] / s, rtol=1e-5, atol=1e-5)
    assert np.allclose(f[:, 3:6], (y[rows] - x0[rows]) / s, rtol=1e-4, atol=1e-4)
    assert np.allclose(t, (xs[rows] - y[rows]) / s, rtol=1e-4, atol=1e-4)
    # edge-vector slots of an interior vertex: +x, +x+z, +z, -x, -x-z, -z
    n = 12
    v = 5 * n + 6
    k = int(np.nonzero(rows == v)[0][0])
    nbrs = [v + 1, v + n + 1, v + n, v - 1, v - n - 1, v - n]
    for q, u in enumerate(nbrs):
        L = np.linalg.norm(inst.positions[u] - inst.positions[v])
        assert np.allclose(f[k, 6 + 3 * q:9 + 3 * q], (x0[u] - x0[v]) / L, rtol=1e-4, atol=1e-5)


def _record(ats, cloth, inst, frames, iters, seed0, ds):
    M = float(inst.mass.sum())
    cloth.set_state(inst.positions, np.zeros_like(inst.positions))
    for f in range(frames):
        cloth.set_accel(configs.wind_accel(np.random.RandomState(seed0 + f), M))
        cloth.predict()
        cloth.record_begin()
        cloth.vbd_iterations(iters)
        cloth.record_end(ds)
        cloth.update_velocity()


def test_training_reduces_loss(ats):
    inst = configs.grid_instance(32)
    cloth = ats.Cloth([inst], implicit_dt=1.0 / 60.0, num_substep=1, iterations=60, damping=2.0)
    ds = ats.Dataset(80 * inst.num_verts)
    _record(ats, cloth, inst, 60, 60, 0, ds)
    m = ats.MLP(seed=0)
    m.fit_normalization(ds)
    f, t = ds.read(0, 4096)
    norm = m.normalization()
    tn = (t - norm[48:51]) / norm[51:54]
    before, _ = m.gradient(f, tn * norm[51:54] + norm[48:51])
    m.train(ds, steps=400, batch=4096, lr=1e-3, seed=1)
    after, _ = m.gradient(f, t)
    assert after < 0.7 * before, (before, after)


def test_fallback_restores_inertial_guess(ats):
    insts, prm = configs.c2(num_instances=3, seed=2, side_range=(10, 20))
    prm = dict(prm, iterations=10)
    a = ats.Cloth(insts, **prm)
    b = ats.Cloth(insts, **prm)
    bad = ats.MLP(seed=9)
    bad.set_params(np.random.RandomState(0).standard_normal(bad.nparams).astype(np.float32) * 3.0)
    norm = bad.normalization()
    norm[51:54] = 50.0  # outputs of tens of gravity steps: the guess raises the potential
    bad.set_normalization(norm)
    for _ in range(3):
        b.frame()
        a.predict()
        used = a.warm_start(bad, fallback=True)
        a.vbd_iterations(10)
        a.update_velocity()
        assert (used == 0).all()
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_learned_warm_start_reaches_plain_residual_in_fewer_iterations(ats):
    """The gain of the network over the inertial guess: iterations the warm-started
    frame needs to reach the residual plain VBD reaches with its full budget."""
    inst = configs.grid_instance(48)
    iters = 100
    cloth = ats.Cloth([inst], implicit_dt=1.0 / 60.0, num_substep=1, iterations=iters, damping=2.0)
    ds = ats.Dataset(260 * inst.num_verts)
    _record(ats, cloth, inst, 120, iters, 0, ds)
    _record(ats, cloth, inst, 120, iters, 1000, ds)
    m = ats.MLP(seed=0)
    m.fit_normalization(ds)
    m.train(ds, steps=1500, batch=8192, lr=1e-3, seed=0)
    m.train(ds, steps=500, batch=8192, lr=3e-4, seed=1)
    M = float(inst.mass.sum())
    cloth.set_state(inst.positions, np.zeros_like(inst.positions))
    needed = []
    for f in range(60):
        cloth.set_accel(configs.wind_accel(np.random.RandomState(10000 + f), M))
        if f >= 30 and f % 3 == 0:
            x0, v0 = cloth.state()
            _, r_plain = cloth.frame_to_residual(0.0, check_every=iters, max_iterations=iters)
            cloth.set_state(x0, v0)
            its, r_warm, used = cloth.frame_warm_to_residual(m, r_plain, check_every=5, max_iterations=iters)
            needed.append(int(its[0]))
            cloth.set_state(x0, v0)
        cloth.frame()
    needed = np.array(needed)
    # the learned guess reaches the plain 100-iteration residual in fewer iterations
    assert np.median(needed) < iters, needed


@pytest.mark.parametrize("n", [40, 181])
def test_tensor_core_inference_matches_tile_forward(ats, n):
    """The frame's inference kernel (tcgen05 MMA, FP32 accumulators in tensor memory,
    128 vertices per tile) against ats_mlp_infer (the shared-memory tile forward that
    is checked against the oracle). Same BF16 quantisation points; the FP32 sums are
    ordered differently (bias after the products), which can move a BF16 rounding, so
    the guesses agree to a tolerance. 181^2 vertices exercise full and partial tiles."""
    inst = configs.grid_instance(n)
    cloth = ats.Cloth([inst], implicit_dt=1.0 / 60.0, num_substep=1, iterations=10, damping=2.0)
    for _ in range(4):
        cloth.frame()
    m = ats.MLP(seed=5)
    m.set_normalization(_norm_vector(np.random.RandomState(2)))
    ds = ats.Dataset(inst.num_verts)
    cloth.predict()
    y = cloth.positions()
    cloth.record_begin()
    cloth.record_end(ds)  # features of the free vertices at this frame start
    f, _ = ds.read()
    cloth.warm_start(m, fallback=False)
    guess = cloth.positions()
    free = np.nonzero(inst.fixed == 0)[0]
    order = cloth.vertex_order()
    rows = np.argsort(order)[np.sort(order[free])]
    s = 9.8 / 3600.0
    out = m.infer(f)
    expect = y[rows] + np.float32(s) * out
    got = (guess[rows] - y[rows]) / np.float32(s)
    err = np.abs(got - out)
    scale = np.max(np.abs(out))
    assert np.linalg.norm(got - out) <= 2e-3 * np.linalg.norm(out), np.linalg.norm(got - out) / np.linalg.norm(out)
    assert np.max(err) <= 2e-2 * scale, (np.max(err), scale)
    assert np.median(err) <= 1e-3 * scale
    assert np.allclose(guess[rows], expect, rtol=0, atol=1e-5)
    pinned = inst.fixed.astype(bool)
    assert np.array_equal(guess[pinned], y[pinned])


def test_warm_frame_graph_equals_eager(ats):
    insts, prm = configs.c2(num_instances=3, seed=4, side_range=(12, 24))
    a = ats.Cloth(insts, **prm)
    b = ats.Cloth(insts, **prm)
    m = ats.MLP(seed=6)
    for _ in range(3):
        a.frame_warm(m, fallback=True, iterations=7, graph=True)
        b.frame_warm(m, fallback=True, iterations=7, graph=False)
    xa, va = a.state()
    xb, vb = b.state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_batch_gradient_and_adam_step(ats):
    # a 3 x 3 grid with only the centre free records one sample per frame, so every
    # batch drawn from the dataset holds copies of that sample
    fixed = np.ones(9, dtype=np.uint8)
    fixed[4] = 0
    inst = configs.grid_instance(3, fixed=fixed)
    cloth = ats.Cloth([inst], implicit_dt=1.0 / 60.0, num_substep=1, iterations=10, damping=2.0)
    ds = ats.Dataset(4)
    cloth.set_accel(np.array([[0.3, -9.8, 0.5]]))
    cloth.predict()
    cloth.record_begin()
    cloth.vbd_iterations(10)
    cloth.record_end(ds)
    assert len(ds) == 1
    rng = np.random.RandomState(6)
    m = ats.MLP(seed=5)
    m.set_normalization(_norm_vector(rng))
    theta0 = m.params()
    f, t = ds.read()
    l1, g1 = m.gradient(f, t)
    # batch 256: the output gradient 2e/(3n) differs from the single sample's by a power
    # of two, so its BF16 rounding is the same and only FP32 summation order remains
    lb, gb = m.batch_gradient(ds, batch=256, seed=7)
    assert np.array_equal(m.params(), theta0)  # a gradient leaves the parameters alone
    assert abs(lb - l1) <= 1e-5 * l1
    assert np.linalg.norm(gb - g1) <= 1e-4 * np.linalg.norm(g1)
    lb2, gb2 = m.batch_gradient(ds, batch=256, seed=7)
    assert lb2 == lb and np.array_equal(gb2, gb)  # deterministic
    # the first Adam step from zero moments moves every parameter by lr * g / (|g| + eps)
    g = rng.standard_normal(theta0.size).astype(np.float32)
    m.apply_gradient(g, lr=1e-3)
    expected = theta0.astype(np.float64) - 1e-3 * g / (np.abs(g) + 1e-8)
    assert np.max(np.abs(m.params() - expected)) < 1e-6
