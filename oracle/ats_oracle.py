"""ctypes wrapper of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of libAtsSim's CPU VBD / XPBD cloth path
(examples/example2_async_iter.cpp, src/Solver/xpbd_constraints.h). Only the
tests, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import this
module, and only as the checker or the timed CPU baseline; the product package
``libatssim_b200`` never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libats_oracle.so")

_lib = None


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("implicit_dt", ctypes.c_float),
        ("num_substep", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("k_stretch", ctypes.c_float),
        ("k_bend", ctypes.c_float),
        ("damping", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("threads", ctypes.c_int),
    ]


def build():
    """Compiles the oracle with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        dp = ctypes.POINTER(ctypes.c_double)
        u8p = ctypes.POINTER(ctypes.c_ubyte)
        L.ato_scene_create.restype = P
        L.ato_scene_create.argtypes = [fp, ctypes.c_int, ip, ctypes.c_int, fp, u8p, ctypes.POINTER(OracleParams)]
        L.ato_scene_destroy.argtypes = [P]
        L.ato_scene_counts.argtypes = [P, ip]
        L.ato_get_edges.argtypes = [P, ip]
        L.ato_get_bending.argtypes = [P, ip]
        L.ato_get_rest.argtypes = [P, fp, fp]
        L.ato_get_coloring.argtypes = [P, ctypes.c_int, ip, ip]
        L.ato_get_adjacency.argtypes = [P, ctypes.c_int, ip, ip]
        L.ato_get_adjacency.restype = ctypes.c_int
        L.ato_set_state.argtypes = [P, fp, fp]
        L.ato_get_state.argtypes = [P, fp, fp]
        L.ato_set_gravity.argtypes = [P, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.ato_frame.argtypes = [P, ctypes.c_int, dp, ctypes.c_int, dp]
        L.ato_run_frames.argtypes = [P, ctypes.c_int, ctypes.c_int]
        L.ato_frame_to_residual.argtypes = [P, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.ato_frame_to_residual.restype = ctypes.c_int
        L.ato_energy_of.argtypes = [P, fp, ctypes.c_int]
        L.ato_energy_of.restype = ctypes.c_double
        L.ato_grad_norm_of.argtypes = [P, fp]
        L.ato_grad_norm_of.restype = ctypes.c_double
        L.ato_grad_norm_pool_of.argtypes = [P, fp]
        L.ato_grad_norm_pool_of.restype = ctypes.c_double
        L.ato_begin_frame.argtypes = [P]
        L.ato_reference_pins.argtypes = [fp, ctypes.c_int, u8p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def reference_pins(positions):
    """Pins of example2:195-209: AABB-normalised z < 0.01 and (x > 0.99 or x < 0.01)."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    out = np.zeros(pos.shape[0], dtype=np.uint8)
    lib().ato_reference_pins(_p(pos, ctypes.c_float), pos.shape[0], _p(out, ctypes.c_ubyte))
    return out


class Scene:
    """One cloth in the oracle: topology, colourings and the CPU solver state."""

    def __init__(self, positions, faces, mass, fixed, *, dt=1.0 / 60.0, substeps=1, iterations=100,
                 k_stretch=1e4, k_bend=2.5e-3, damping=2.0, gravity=(0.0, -9.8, 0.0), threads=1):
        self.positions = np.ascontiguousarray(positions, dtype=np.float32)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        self.mass = np.ascontiguousarray(mass, dtype=np.float32)
        self.fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
        self.nv = self.positions.shape[0]
        prm = OracleParams(dt, substeps, iterations, k_stretch, k_bend, damping,
                           (ctypes.c_float * 3)(*gravity), threads)
        self.params = prm
        self.iterations = iterations
        self.h = lib().ato_scene_create(_p(self.positions, ctypes.c_float), self.nv,
                                        _p(self.faces, ctypes.c_int), self.faces.shape[0],
                                        _p(self.mass, ctypes.c_float), _p(self.fixed, ctypes.c_ubyte),
                                        ctypes.byref(prm))
        c = np.zeros(6, dtype=np.int32)
        lib().ato_scene_counts(self.h, _p(c, ctypes.c_int))
        self.ne, self.nb, self.n_vcolors, self.n_scolors, self.n_bcolors, self.threads = (int(v) for v in c)

    def close(self):
        if self.h:
            lib().ato_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # topology ---------------------------------------------------------
    def edges(self):
        out = np.zeros((self.ne, 2), dtype=np.int32)
        lib().ato_get_edges(self.h, _p(out, ctypes.c_int))
        return out

    def bending_edges(self):
        out = np.zeros((self.nb, 4), dtype=np.int32)
        lib().ato_get_bending(self.h, _p(out, ctypes.c_int))
        return out

    def rest(self):
        L = np.zeros(self.ne, dtype=np.float32)
        Q = np.zeros((self.nb, 4, 4), dtype=np.float32)  # Q[e, col, row]
        lib().ato_get_rest(self.h, _p(L, ctypes.c_float), _p(Q, ctypes.c_float))
        return L, Q

    def coloring(self, which):
        """which: 'vertex', 'stretch' or 'bending' -> list of int32 arrays."""
        w = {"vertex": 0, "stretch": 1, "bending": 2}[which]
        n = {0: self.n_vcolors, 1: self.n_scolors, 2: self.n_bcolors}[w]
        total = {0: self.nv, 1: self.ne, 2: self.nb}[w]
        prefix = np.zeros(n + 1, dtype=np.int32)
        items = np.zeros(max(total, 1), dtype=np.int32)
        lib().ato_get_coloring(self.h, w, _p(prefix, ctypes.c_int), _p(items, ctypes.c_int))
        return [items[prefix[c]:prefix[c + 1]].copy() for c in range(n)]

    def adjacency(self, which):
        """which: 'verts_bending', 'edges' or 'bending' -> (prefix, items) CSR."""
        w = {"verts_bending": 0, "edges": 1, "bending": 2}[which]
        n = lib().ato_get_adjacency(self.h, w, None, None)
        prefix = np.zeros(self.nv + 1, dtype=np.int32)
        items = np.zeros(max(n, 1), dtype=np.int32)
        lib().ato_get_adjacency(self.h, w, _p(prefix, ctypes.c_int), _p(items, ctypes.c_int))
        return prefix, items[:n]

    # state -------------------------------------------------------------
    def set_state(self, x, v):
        x = np.ascontiguousarray(x, dtype=np.float32)
        v = np.ascontiguousarray(v, dtype=np.float32)
        lib().ato_set_state(self.h, _p(x, ctypes.c_float), _p(v, ctypes.c_float))

    def state(self):
        x = np.zeros((self.nv, 3), dtype=np.float32)
        v = np.zeros((self.nv, 3), dtype=np.float32)
        lib().ato_get_state(self.h, _p(x, ctypes.c_float), _p(v, ctypes.c_float))
        return x, v

    def set_gravity(self, g):
        lib().ato_set_gravity(self.h, float(g[0]), float(g[1]), float(g[2]))

    def frame(self, solver="vbd", log_energy=False, with_bending=False, log_residual=False):
        """Runs one frame; returns (energy_log, residual_log) (None when not requested)."""
        s = 0 if solver == "vbd" else 1
        e = np.zeros(self.iterations + 1, dtype=np.float64) if log_energy else None
        r = np.zeros(self.iterations + 1, dtype=np.float64) if log_residual else None
        lib().ato_frame(self.h, s, _p(e, ctypes.c_double) if e is not None else None, int(with_bending),
                        _p(r, ctypes.c_double) if r is not None else None)
        return e, r

    def frame_to_residual(self, tol, check_every=10, max_iterations=1000, policy=0):
        """One VBD frame iterated until ||grad G(x)|| <= tol ||grad G(y)||, probed every
        check_every iterations (policy 0) or on the extrapolated schedule (policy 1), and
        at max_iterations -> (iterations, relative residual)."""
        r = ctypes.c_double(0.0)
        it = lib().ato_frame_to_residual(self.h, float(tol), int(check_every), int(max_iterations), int(policy),
                                         ctypes.byref(r))
        return int(it), float(r.value)

    def run(self, frames, solver="vbd"):
        lib().ato_run_frames(self.h, 0 if solver == "vbd" else 1, frames)

    def begin_frame(self):
        lib().ato_begin_frame(self.h)

    def energy_of(self, x, with_bending=True):
        x = np.ascontiguousarray(x, dtype=np.float32)
        return lib().ato_energy_of(self.h, _p(x, ctypes.c_float), int(with_bending))

    def grad_norm_pool_of(self, x):
        """grad_norm_of gathered per vertex on the thread pool (the to-residual probe)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        return lib().ato_grad_norm_pool_of(self.h, _p(x, ctypes.c_float))

    def grad_norm_of(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        return lib().ato_grad_norm_of(self.h, _p(x, ctypes.c_float))


def async_merge(begin, mine, other, weight):
    """Core::read_and_solve_conflict (src/Solver/xpbd_constraints.h:815-869) over all
    vertices, in FP32 with one rounding per operation in the reference's order:
    returns the merged positions (the new iterate and fork point of "mine")."""
    f = np.float32
    b, s, o = (np.asarray(a, dtype=np.float32).reshape(-1, 3) for a in (begin, mine, other))
    w = f(weight)
    if w > f(1.19209290e-7):
        ds = (s - b).astype(np.float32)
        do = (o - b).astype(np.float32)

        def moved(d):
            sq = (d * d).astype(np.float32)
            return ((sq[:, 0] + sq[:, 1]).astype(np.float32) + sq[:, 2]).astype(np.float32) != 0

        a_s, a_o = moved(ds), moved(do)
        both = (b + (w * (ds + do).astype(np.float32)).astype(np.float32)).astype(np.float32)
        out = b.copy()
        out[a_s & a_o] = both[a_s & a_o]
        only_s = a_s & ~a_o
        only_o = a_o & ~a_s
        out[only_s] = s[only_s]
        out[only_o] = o[only_o]
        return out
    return (f(0.5) * (s + o).astype(np.float32)).astype(np.float32)
