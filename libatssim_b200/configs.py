"""Workload builders for the cloth solver's benchmark and parity configurations.

Every mesh is synthetic and seeded; nothing is read from disk.

  c0  64 x 64 grid, 1 m x 1 m, uniform diagonal split, k = 1e3 N/m, k_b = 1e-2,
      0.1 kg area-lumped, two top corners pinned, h = 1/60, 100 VBD iterations.
  c1  512 x 512 grid, same material and pinning, 50 iterations per frame.
  c2  256 instances, side U{16..256}, k log-uniform [1e2, 1e4], k_b log-uniform
      [1e-3, 1e-1], 1-4 random boundary pins, 50 iterations per frame.
  reference_square  square8K-style reference setup: 0.01 kg per vertex, k = 1e4,
      k_b = 5e-3 * 0.5, reference pin rule (examples/example2_async_iter.cpp:195-225,
      715-749).
"""
import numpy as np

from . import GRID_UNIFORM, Instance, grid_mesh, mass_area_weighted, reference_pins

MATERIAL = dict(k_stretch=1e3, k_bend=1e-2, total_mass=0.1)


def corner_pins(n):
    """The two corners of the grid row with the smallest z (row 0)."""
    fixed = np.zeros(n * n, dtype=np.uint8)
    fixed[0] = 1
    fixed[n - 1] = 1
    return fixed


def grid_instance(n, k_stretch=MATERIAL["k_stretch"], k_bend=MATERIAL["k_bend"], total_mass=MATERIAL["total_mass"],
                  fixed=None, pattern=GRID_UNIFORM):
    pos, faces = grid_mesh(n, pattern)
    mass = mass_area_weighted(pos, faces, total_mass)
    if fixed is None:
        fixed = corner_pins(n)
    return Instance(pos, faces, mass, fixed, k_stretch, k_bend)


def c0():
    return [grid_instance(64)], dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=100, damping=2.0)


def c1():
    return [grid_instance(512)], dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=50, damping=2.0)


def boundary_vertices(n):
    r = np.arange(n)
    ids = np.concatenate([r, (n - 1) * n + r, r[1:-1] * n, r[1:-1] * n + n - 1])
    return np.unique(ids)


def c2(num_instances=256, seed=0, side_range=(16, 256)):
    """Batched instances of uneven size; instance i draws from RandomState(seed + i)."""
    insts = []
    for i in range(num_instances):
        rng = np.random.RandomState(seed + i)
        n = int(rng.randint(side_range[0], side_range[1] + 1))
        k = float(10 ** rng.uniform(2.0, 4.0))
        kb = float(10 ** rng.uniform(-3.0, -1.0))
        npins = int(rng.randint(1, 5))
        fixed = np.zeros(n * n, dtype=np.uint8)
        fixed[rng.choice(boundary_vertices(n), size=npins, replace=False)] = 1
        insts.append(grid_instance(n, k_stretch=k, k_bend=kb, fixed=fixed))
    return insts, dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=50, damping=2.0)


def wind_accel(rng, total_mass, gravity=(0.0, -9.8, 0.0), max_force=2.0):
    """Gravity plus a random wind force: direction uniform on the sphere, magnitude
    U[0, max_force] N, spread over the instance mass."""
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    f = rng.uniform(0.0, max_force) * d
    return np.asarray(gravity, dtype=np.float64) + f / float(total_mass)


def c3():
    """128 x 128 cloth of the c0 material, random wind per frame, 200 iterations."""
    return [grid_instance(128)], dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=200, damping=2.0)


def c4(num_instances=64, seed=0, side_range=(64, 512)):
    """Batched instances of the c0 material, side U{64..512} from RandomState(seed + i),
    two top corners pinned; random wind per instance per frame; 50 iterations."""
    insts = []
    for i in range(num_instances):
        rng = np.random.RandomState(seed + i)
        insts.append(grid_instance(int(rng.randint(side_range[0], side_range[1] + 1))))
    return insts, dict(implicit_dt=1.0 / 60.0, num_substep=1, iterations=50, damping=2.0)


def reference_square(positions, faces):
    """libAtsSim Example 2 material on a given mesh (0.01 kg per vertex)."""
    mass = np.full(positions.shape[0], 0.01, dtype=np.float32)
    return [Instance(positions, faces, mass, reference_pins(positions), 1e4, 5e-3 * 0.5)], dict(
        implicit_dt=1.0 / 60.0, num_substep=1, iterations=100, damping=2.0)
