"""The oracle's residual probe and to-residual frame (CPU only)."""
import numpy as np

from libatssim_b200 import configs


def _scene(oracle, n=24, iterations=20):
    inst = configs.grid_instance(n)
    return inst, oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, iterations=iterations,
                              k_stretch=inst.k_stretch, k_bend=inst.k_bend, threads=2)


def test_pooled_gradient_norm_equals_serial(oracle):
    inst, s = _scene(oracle)
    for _ in range(3):
        s.frame()
    s.begin_frame()
    x, _ = s.state()
    x = x + 1e-3 * np.random.RandomState(0).standard_normal(x.shape).astype(np.float32)
    a, b = s.grad_norm_of(x), s.grad_norm_pool_of(x)
    assert abs(a - b) <= 1e-12 * a


def test_frame_to_residual_probes_and_cap(oracle):
    inst, s = _scene(oracle)
    s.frame()
    x, v = s.state()
    # tol 0 never stops early: the cap, even when it is not a multiple of check_every
    it, r = s.frame_to_residual(0.0, check_every=4, max_iterations=10)
    assert it == 10 and 0.0 < r < 1.0
    # a loose tolerance stops at the first probe
    s.set_state(x, v)
    it, r = s.frame_to_residual(10.0, check_every=4, max_iterations=10)
    assert it == 4
    # the same frame as the fixed-iteration one when the cap is reached
    _, s2 = _scene(oracle, iterations=10)
    s2.set_state(x, v)
    s2.frame()
    s.set_state(x, v)
    s.frame_to_residual(0.0, check_every=3, max_iterations=10)
    assert np.array_equal(s.state()[0], s2.state()[0])
