"""libatssim_b200 -- B200-native cloth solver (VBD and XPBD) behind a C ABI.

Python access to ``libats_b200.so`` (include/ats_cloth.h) through ctypes. The
compute path is the CUDA library; this module only marshals arrays and status
codes. Loading fails loudly when the library is missing: there is no CPU path.

Names follow libAtsSim: a *cloth* holds one or more instances (meshes), each with
its own stiffness; a *frame* is predict -> iterations x colours -> update
(examples/example2_async_iter.cpp:1082-1143).
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libats_b200.so")

ATS_OK, ATS_ERR_INVALID, ATS_ERR_CUDA, ATS_ERR_NOMEM, ATS_ERR_TIMEOUT, ATS_ERR_STATE = range(6)
SOLVER_VBD, SOLVER_XPBD = 0, 1
GRID_UNIFORM, GRID_ALTERNATING = 0, 1
COLORING = {"vertex": 0, "stretch": 1, "bending": 2}


class AtsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"ats status {status}: {msg}")
        self.status = status


class InstanceDesc(ctypes.Structure):
    _fields_ = [
        ("num_verts", ctypes.c_int),
        ("positions", ctypes.POINTER(ctypes.c_float)),
        ("num_faces", ctypes.c_int),
        ("faces", ctypes.POINTER(ctypes.c_int)),
        ("mass", ctypes.POINTER(ctypes.c_float)),
        ("fixed", ctypes.POINTER(ctypes.c_ubyte)),
        ("k_stretch", ctypes.c_float),
        ("k_bend", ctypes.c_float),
    ]


class SolverParams(ctypes.Structure):
    _fields_ = [
        ("implicit_dt", ctypes.c_float),
        ("num_substep", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("damping", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("threads_per_vertex", ctypes.c_int),
        ("block_size", ctypes.c_int),
    ]


class ClothInfo(ctypes.Structure):
    _fields_ = [
        ("num_instances", ctypes.c_int),
        ("num_verts", ctypes.c_int),
        ("num_edges", ctypes.c_int),
        ("num_bending_edges", ctypes.c_int),
        ("num_vertex_colors", ctypes.c_int),
        ("num_stretch_colors", ctypes.c_int),
        ("num_bending_colors", ctypes.c_int),
        ("threads_per_vertex", ctypes.c_int),
        ("block_size", ctypes.c_int),
        ("stencil_slots", ctypes.c_int),
        ("device_bytes", ctypes.c_longlong),
        ("vbd_form", ctypes.c_int),
        ("xpbd_form", ctypes.c_int),
        ("list_form", ctypes.c_int),
        ("sweep_layout_bytes", ctypes.c_longlong),
        ("tune_source", ctypes.c_int),
        ("l2_persisting", ctypes.c_int),
    ]


_lib = None
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_ubyte)
_vp = ctypes.c_void_p

# (name, argtypes) of every exported C entry point; all return int unless noted.
_SIGNATURES = {
    "ats_grid_mesh": [ctypes.c_int, ctypes.c_int, _fp, _ip],
    "ats_reference_pins": [_fp, ctypes.c_int, _u8p],
    "ats_mass_area_weighted": [_fp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_float, _fp],
    "ats_obj_read": [ctypes.c_char_p, _ip, _fp, _ip, _ip],
    "ats_obj_write": [ctypes.c_char_p, _fp, ctypes.c_int, _ip, ctypes.c_int],
    "ats_state_write": [ctypes.c_char_p, _fp, _fp, ctypes.c_int, ctypes.c_int],
    "ats_state_read": [ctypes.c_char_p, _fp, _fp, _ip, _ip],
    "ats_topology_build": [ctypes.POINTER(InstanceDesc), ctypes.POINTER(_vp)],
    "ats_topology_destroy": [_vp],
    "ats_topology_counts": [_vp, _ip],
    "ats_topology_edges": [_vp, _ip, _ip],
    "ats_topology_rest": [_vp, _fp, _fp],
    "ats_topology_coloring": [_vp, ctypes.c_int, _ip, _ip],
    "ats_cloth_create": [ctypes.POINTER(InstanceDesc), ctypes.c_int, ctypes.POINTER(SolverParams), ctypes.POINTER(_vp)],
    "ats_cloth_destroy": [_vp],
    "ats_cloth_query": [_vp, ctypes.POINTER(ClothInfo)],
    "ats_cloth_vertex_order": [_vp, _ip],
    "ats_set_state": [_vp, _fp, _fp, _vp],
    "ats_get_state": [_vp, _fp, _fp, _vp],
    "ats_get_positions": [_vp, _fp, _vp],
    "ats_set_positions": [_vp, _fp, _vp],
    "ats_set_accel": [_vp, _fp, _vp],
    "ats_predict_position": [_vp, _vp],
    "ats_vbd_color_sweep": [_vp, ctypes.c_int, _vp],
    "ats_vbd_iterations": [_vp, ctypes.c_int, _vp],
    "ats_update_velocity": [_vp, _vp],
    "ats_xpbd_reset_constraints": [_vp, _vp],
    "ats_xpbd_stretch_color": [_vp, ctypes.c_int, _vp],
    "ats_xpbd_bending_color": [_vp, ctypes.c_int, _vp],
    "ats_frame": [_vp, ctypes.c_int, _vp],
    "ats_frame_graph": [_vp, ctypes.c_int, _vp],
    "ats_autotune": [_vp, ctypes.c_int, _vp, _ip, _ip],
    "ats_energy": [_vp, _dp, _vp],
    "ats_frame_to_residual": [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _ip, _dp, _vp],
    "ats_residual": [_vp, _dp, _vp],
    "ats_potential": [_vp, _dp, _vp],
    "ats_async_fork": [_vp, _vp],
    "ats_async_merge": [_vp, _fp, ctypes.c_float, _vp],
    "ats_mlp_create": [ctypes.c_ulonglong, ctypes.POINTER(_vp)],
    "ats_mlp_destroy": [_vp],
    "ats_mlp_get_params": [_vp, _fp],
    "ats_mlp_set_params": [_vp, _fp],
    "ats_mlp_infer": [_vp, _fp, ctypes.c_int, _fp, _vp],
    "ats_mlp_get_normalization": [_vp, _fp],
    "ats_mlp_set_normalization": [_vp, _fp],
    "ats_mlp_fit_normalization": [_vp, _vp, _vp],
    "ats_mlp_gradient": [_vp, _fp, _fp, ctypes.c_int, _fp, _fp, _vp],
    "ats_mlp_batch_gradient": [_vp, _vp, ctypes.c_int, ctypes.c_ulonglong, _fp, _fp, _vp],
    "ats_mlp_apply_gradient": [_vp, _fp, ctypes.c_float, _vp],
    "ats_dataset_create": [ctypes.c_longlong, ctypes.POINTER(_vp)],
    "ats_dataset_destroy": [_vp],
    "ats_dataset_size": [_vp, ctypes.POINTER(ctypes.c_longlong)],
    "ats_dataset_read": [_vp, ctypes.c_longlong, ctypes.c_longlong, _fp, _fp],
    "ats_record_frame_begin": [_vp, _vp],
    "ats_record_frame_end": [_vp, _vp, _vp],
    "ats_mlp_train": [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_ulonglong, _fp, _vp],
    "ats_warm_start": [_vp, _vp, ctypes.c_int, _ip, _vp],
    "ats_frame_warm": [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp],
    "ats_frame_warm_to_residual": [_vp, _vp, ctypes.c_int, ctypes.c_double, _dp, _ip, ctypes.c_int, ctypes.c_int, _ip,
                                   _dp, _ip, _vp],
    "ats_frame_to_residuals": [_vp, _dp, _ip, ctypes.c_int, ctypes.c_int, _ip, _dp, _vp],
    "ats_kernel_launches": [ctypes.POINTER(ctypes.c_longlong)],
    "ats_set_probe_policy": [_vp, ctypes.c_int],
    "ats_set_sweep_form": [_vp, ctypes.c_int, ctypes.c_int],
    "ats_set_list_sweep": [_vp, ctypes.c_int],
    "ats_set_l2_persisting": [_vp, ctypes.c_int],
    "ats_selftest_bounded_waits": [ctypes.c_uint, _ip, _ip],
    "ats_autotune_cache_size": [],
    "ats_autotune_cache_save": [ctypes.c_char_p],
    "ats_autotune_cache_load": [ctypes.c_char_p],
    "ats_energy_noalloc": [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int,
                           ctypes.c_float, ctypes.c_float, _fp, ctypes.c_float, _vp, _vp],
}


def lib():
    """Loads libats_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m libatssim_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.ats_last_error.restype = ctypes.c_char_p
        L.ats_last_error.argtypes = []
        L.ats_mlp_param_count.restype = ctypes.c_int
        L.ats_mlp_param_count.argtypes = []
        L.ats_autotune_cache_clear.restype = None
        L.ats_autotune_cache_clear.argtypes = []
        _lib = L
    return _lib


def _check(status):
    if status != ATS_OK:
        raise AtsError(status, lib().ats_last_error().decode())


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _stream(stream):
    """Accepts None, an int handle or a torch.cuda.Stream."""
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def energy_noalloc(x, x_start, v, mass, fixed, num_verts, edges, rest_length, num_edges, bending, q,
                   num_bending_edges, k_stretch, k_bend, accel, h, out3, stream=None):
    """ats_energy_noalloc: FP64 energy terms of plain device arrays (all array
    arguments are device addresses as ints) into the device array out3, using only
    the library's static scratch (no device allocation). Enqueues on `stream`."""
    acc = np.ascontiguousarray(accel, dtype=np.float32)
    _check(lib().ats_energy_noalloc(x, x_start, v, mass, fixed, int(num_verts), edges, rest_length, int(num_edges),
                                    bending, q, int(num_bending_edges), float(k_stretch), float(k_bend),
                                    _p(acc, ctypes.c_float), float(h), out3, _stream(stream)))


def kernel_launches():
    """Kernels launched by the library so far in this process (direct launches plus
    the kernel nodes of CUDA-graph replays)."""
    n = ctypes.c_longlong(0)
    _check(lib().ats_kernel_launches(ctypes.byref(n)))
    return int(n.value)


def selftest_bounded_waits(polls=4096):
    """Runs a grid-barrier wait and an mbarrier wait that cannot complete; returns their
    statuses (ATS_ERR_TIMEOUT each when the bound worked) (ats_selftest_bounded_waits)."""
    b, m = ctypes.c_int(-1), ctypes.c_int(-1)
    _check(lib().ats_selftest_bounded_waits(int(polls), ctypes.byref(b), ctypes.byref(m)))
    return b.value, m.value


def autotune_cache_size():
    """Entries of the process's autotuning cache (one per GPU and mesh class)."""
    return int(lib().ats_autotune_cache_size())


def autotune_cache_clear():
    lib().ats_autotune_cache_clear()


def autotune_cache_save(path):
    _check(lib().ats_autotune_cache_save(os.fsencode(path)))


def autotune_cache_load(path):
    """Merges a file written by autotune_cache_save into the cache."""
    _check(lib().ats_autotune_cache_load(os.fsencode(path)))


# ---------------------------------------------------------------- mesh helpers
def grid_mesh(n, pattern=GRID_UNIFORM):
    """n x n grid on y = 0 over [-0.5, 0.5]^2 -> (positions (n*n, 3), faces (2(n-1)^2, 3))."""
    pos = np.zeros((n * n, 3), dtype=np.float32)
    faces = np.zeros((2 * (n - 1) * (n - 1), 3), dtype=np.int32)
    _check(lib().ats_grid_mesh(n, pattern, _p(pos, ctypes.c_float), _p(faces, ctypes.c_int)))
    return pos, faces


def reference_pins(positions):
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    out = np.zeros(pos.shape[0], dtype=np.uint8)
    _check(lib().ats_reference_pins(_p(pos, ctypes.c_float), pos.shape[0], _p(out, ctypes.c_ubyte)))
    return out


def mass_area_weighted(positions, faces, total_mass):
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    out = np.zeros(pos.shape[0], dtype=np.float32)
    _check(lib().ats_mass_area_weighted(_p(pos, ctypes.c_float), pos.shape[0], _p(f, ctypes.c_int), f.shape[0],
                                        float(total_mass), _p(out, ctypes.c_float)))
    return out


def obj_read(path):
    nv, nf = ctypes.c_int(0), ctypes.c_int(0)
    _check(lib().ats_obj_read(path.encode(), ctypes.byref(nv), None, ctypes.byref(nf), None))
    pos = np.zeros((nv.value, 3), dtype=np.float32)
    faces = np.zeros((nf.value, 3), dtype=np.int32)
    _check(lib().ats_obj_read(path.encode(), ctypes.byref(nv), _p(pos, ctypes.c_float), ctypes.byref(nf),
                              _p(faces, ctypes.c_int)))
    return pos, faces


def obj_write(path, positions, faces):
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    _check(lib().ats_obj_write(path.encode(), _p(pos, ctypes.c_float), pos.shape[0], _p(f, ctypes.c_int), f.shape[0]))


def state_write(path, x, v, frame=0):
    x = np.ascontiguousarray(x, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    _check(lib().ats_state_write(path.encode(), _p(x, ctypes.c_float), _p(v, ctypes.c_float), x.shape[0], int(frame)))


def state_read(path):
    """-> (x, v, frame)"""
    n, fr = ctypes.c_int(0), ctypes.c_int(0)
    _check(lib().ats_state_read(path.encode(), None, None, ctypes.byref(n), ctypes.byref(fr)))
    x = np.zeros((n.value, 3), dtype=np.float32)
    v = np.zeros((n.value, 3), dtype=np.float32)
    _check(lib().ats_state_read(path.encode(), _p(x, ctypes.c_float), _p(v, ctypes.c_float), ctypes.byref(n),
                                ctypes.byref(fr)))
    return x, v, fr.value


class Instance:
    """One cloth mesh with its material: positions (V,3), faces (F,3), mass (V,),
    fixed (V,), k_stretch, k_bend (effective quadratic bending stiffness)."""

    def __init__(self, positions, faces, mass, fixed, k_stretch, k_bend):
        self.positions = np.ascontiguousarray(positions, dtype=np.float32)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        self.mass = np.ascontiguousarray(mass, dtype=np.float32)
        self.fixed = np.ascontiguousarray(fixed, dtype=np.uint8)
        self.k_stretch = float(k_stretch)
        self.k_bend = float(k_bend)

    @property
    def num_verts(self):
        return self.positions.shape[0]

    def desc(self):
        return InstanceDesc(self.num_verts, _p(self.positions, ctypes.c_float), self.faces.shape[0],
                            _p(self.faces, ctypes.c_int), _p(self.mass, ctypes.c_float),
                            _p(self.fixed, ctypes.c_ubyte), self.k_stretch, self.k_bend)


class Topology:
    """Host-only topology of one instance (edges, bending edges, colourings, rest state)."""

    def __init__(self, inst):
        self._inst = inst
        d = inst.desc()
        h = _vp()
        _check(lib().ats_topology_build(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        c = np.zeros(5, dtype=np.int32)
        _check(lib().ats_topology_counts(self.h, _p(c, ctypes.c_int)))
        self.ne, self.nb, self.n_vcolors, self.n_scolors, self.n_bcolors = (int(v) for v in c)

    def __del__(self):
        try:
            if self.h:
                lib().ats_topology_destroy(self.h)
        except Exception:
            pass

    def edges(self):
        e = np.zeros((self.ne, 2), dtype=np.int32)
        b = np.zeros((self.nb, 4), dtype=np.int32)
        _check(lib().ats_topology_edges(self.h, _p(e, ctypes.c_int), _p(b, ctypes.c_int)))
        return e, b

    def rest(self):
        L = np.zeros(self.ne, dtype=np.float32)
        Q = np.zeros((self.nb, 4, 4), dtype=np.float32)
        _check(lib().ats_topology_rest(self.h, _p(L, ctypes.c_float), _p(Q, ctypes.c_float)))
        return L, Q

    def coloring(self, which):
        w = COLORING[which]
        n = {0: self.n_vcolors, 1: self.n_scolors, 2: self.n_bcolors}[w]
        total = {0: self._inst.num_verts, 1: self.ne, 2: self.nb}[w]
        prefix = np.zeros(n + 1, dtype=np.int32)
        items = np.zeros(max(total, 1), dtype=np.int32)
        _check(lib().ats_topology_coloring(self.h, w, _p(prefix, ctypes.c_int), _p(items, ctypes.c_int)))
        return [items[prefix[c]:prefix[c + 1]].copy() for c in range(n)]


class Cloth:
    """A solver handle over one or more instances (ats_cloth_create)."""

    def __init__(self, instances, *, implicit_dt=1.0 / 60.0, num_substep=1, iterations=100, damping=2.0,
                 gravity=(0.0, -9.8, 0.0), threads_per_vertex=0, block_size=0):
        if isinstance(instances, Instance):
            instances = [instances]
        self.instances = list(instances)
        descs = (InstanceDesc * len(self.instances))(*[i.desc() for i in self.instances])
        self.params = SolverParams(implicit_dt, num_substep, iterations, damping,
                                   (ctypes.c_float * 3)(*gravity), threads_per_vertex, block_size)
        h = _vp()
        _check(lib().ats_cloth_create(descs, len(self.instances), ctypes.byref(self.params), ctypes.byref(h)))
        self.h = h
        info = ClothInfo()
        _check(lib().ats_cloth_query(self.h, ctypes.byref(info)))
        self.info = info
        self.nv = info.num_verts
        self.iterations = iterations

    def close(self):
        if getattr(self, "h", None):
            lib().ats_cloth_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def vertex_order(self):
        """layout_of_caller: device position of every caller vertex."""
        out = np.zeros(self.nv, dtype=np.int32)
        _check(lib().ats_cloth_vertex_order(self.h, _p(out, ctypes.c_int)))
        return out

    # state -------------------------------------------------------------
    def set_state(self, x, v=None, stream=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float32)
        _check(lib().ats_set_state(self.h, _p(x, ctypes.c_float), None if vv is None else _p(vv, ctypes.c_float),
                                   _stream(stream)))

    def state(self, stream=None):
        x = np.zeros((self.nv, 3), dtype=np.float32)
        v = np.zeros((self.nv, 3), dtype=np.float32)
        _check(lib().ats_get_state(self.h, _p(x, ctypes.c_float), _p(v, ctypes.c_float), _stream(stream)))
        return x, v

    def async_fork(self, stream=None):
        """The current iterate becomes the fork point of two-device iteration."""
        _check(lib().ats_async_fork(self.h, _stream(stream)))

    def async_merge(self, other_positions, weight=0.5, stream=None):
        """Merges another device's iterate (caller order) into this one
        (Core::read_and_solve_conflict); the result is also the new fork point."""
        o = np.ascontiguousarray(other_positions, dtype=np.float32)
        _check(lib().ats_async_merge(self.h, _p(o, ctypes.c_float), float(weight), _stream(stream)))

    def state_into(self, x, v, stream=None):
        """ats_get_state into caller arrays (C-contiguous float32 (V, 3), e.g. views of
        pinned host memory, which the copies then reach at full bus speed)."""
        for a in (x, v):
            if a.dtype != np.float32 or not a.flags.c_contiguous or a.shape != (self.nv, 3):
                raise ValueError("state_into needs C-contiguous float32 arrays of shape (num_verts, 3)")
        _check(lib().ats_get_state(self.h, _p(x, ctypes.c_float), _p(v, ctypes.c_float), _stream(stream)))

    def positions(self, stream=None):
        x = np.zeros((self.nv, 3), dtype=np.float32)
        _check(lib().ats_get_positions(self.h, _p(x, ctypes.c_float), _stream(stream)))
        return x

    def set_positions(self, x, stream=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        _check(lib().ats_set_positions(self.h, _p(x, ctypes.c_float), _stream(stream)))

    def set_accel(self, accel, stream=None):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(accel, dtype=np.float32), (self.info.num_instances, 3)))
        _check(lib().ats_set_accel(self.h, _p(a, ctypes.c_float), _stream(stream)))

    # steps ---------------------------------------------------------------
    def predict(self, stream=None):
        _check(lib().ats_predict_position(self.h, _stream(stream)))

    def vbd_color_sweep(self, color, stream=None):
        _check(lib().ats_vbd_color_sweep(self.h, int(color), _stream(stream)))

    def vbd_iterations(self, n, stream=None):
        _check(lib().ats_vbd_iterations(self.h, int(n), _stream(stream)))

    def autotune(self, iterations=10, stream=None):
        """Picks lanes-per-vertex and block size by timing; returns (tpv, block)."""
        t, b = ctypes.c_int(0), ctypes.c_int(0)
        _check(lib().ats_autotune(self.h, int(iterations), _stream(stream), ctypes.byref(t), ctypes.byref(b)))
        info = ClothInfo()
        _check(lib().ats_cloth_query(self.h, ctypes.byref(info)))
        self.info = info
        return t.value, b.value

    def update_velocity(self, stream=None):
        _check(lib().ats_update_velocity(self.h, _stream(stream)))

    def xpbd_reset(self, stream=None):
        _check(lib().ats_xpbd_reset_constraints(self.h, _stream(stream)))

    def xpbd_stretch_color(self, color, stream=None):
        _check(lib().ats_xpbd_stretch_color(self.h, int(color), _stream(stream)))

    def xpbd_bending_color(self, color, stream=None):
        _check(lib().ats_xpbd_bending_color(self.h, int(color), _stream(stream)))

    def frame(self, solver=SOLVER_VBD, stream=None, graph=False):
        fn = lib().ats_frame_graph if graph else lib().ats_frame
        _check(fn(self.h, solver, _stream(stream)))

    def frame_warm(self, mlp, fallback=True, iterations=-1, graph=False, stream=None):
        _check(lib().ats_frame_warm(self.h, mlp.h, int(fallback), int(iterations), int(graph), _stream(stream)))

    def warm_start(self, mlp, fallback=True, stream=None):
        used = np.zeros(self.info.num_instances, dtype=np.int32)
        _check(lib().ats_warm_start(self.h, mlp.h, int(fallback), _p(used, ctypes.c_int), _stream(stream)))
        return used

    def frame_warm_to_residual(self, mlp, tol, fallback=True, check_every=10, max_iterations=1000, first_check=None,
                               stream=None):
        """frame_to_residual with the learned guess; tol is a float or one value per
        instance, first_check None or one first-probe iteration per instance; returns
        (iterations, residual, used)."""
        n = self.info.num_instances
        it = np.zeros(n, dtype=np.int32)
        res = np.zeros(n, dtype=np.float64)
        used = np.zeros(n, dtype=np.int32)
        tols = None if np.isscalar(tol) else np.ascontiguousarray(tol, dtype=np.float64)
        fc = None if first_check is None else np.ascontiguousarray(first_check, dtype=np.int32)
        _check(lib().ats_frame_warm_to_residual(self.h, mlp.h, int(fallback), float(tol) if tols is None else 0.0,
                                                None if tols is None else _p(tols, ctypes.c_double),
                                                None if fc is None else _p(fc, ctypes.c_int), int(check_every),
                                                int(max_iterations), _p(it, ctypes.c_int), _p(res, ctypes.c_double),
                                                _p(used, ctypes.c_int), _stream(stream)))
        return it, res, used

    def record_begin(self, stream=None):
        _check(lib().ats_record_frame_begin(self.h, _stream(stream)))

    def record_end(self, dataset, stream=None):
        _check(lib().ats_record_frame_end(self.h, dataset.h, _stream(stream)))

    def set_sweep_form(self, form, solver=SOLVER_VBD):
        """Iterations of fixed-iteration frames of `solver`: 0 one launch per colour, 1
        one persistent cooperative launch (ats_set_sweep_form)."""
        _check(lib().ats_set_sweep_form(self.h, int(solver), int(form)))
        info = ClothInfo()
        _check(lib().ats_cloth_query(self.h, ctypes.byref(info)))
        self.info = info

    def set_list_sweep(self, form):
        """Sweep of the residual-driven frames: 0 plain, 1 pipelined, 2 streamed
        (ats_set_list_sweep)."""
        _check(lib().ats_set_list_sweep(self.h, int(form)))
        info = ClothInfo()
        _check(lib().ats_cloth_query(self.h, ctypes.byref(info)))
        self.info = info

    def set_l2_persisting(self, on):
        """List sweeps keep the positions in L2 as persisting lines (ats_set_l2_persisting)."""
        _check(lib().ats_set_l2_persisting(self.h, int(bool(on))))
        info = ClothInfo()
        _check(lib().ats_cloth_query(self.h, ctypes.byref(info)))
        self.info = info

    def set_probe_policy(self, policy):
        """Probe schedule of the residual-driven frames: 0 fixed period, 1 extrapolated
        from the residual's contraction (ats_set_probe_policy)."""
        _check(lib().ats_set_probe_policy(self.h, int(policy)))

    def frame_to_residual(self, tol, check_every=10, max_iterations=1000, first_check=None, stream=None):
        """One frame iterated until every instance reaches ||grad G|| <= tol ||grad G(y)||
        (or max_iterations); tol is a float or one value per instance, first_check None
        or one first-probe iteration per instance; returns (iterations per instance,
        relative residual per instance)."""
        n = self.info.num_instances
        it = np.zeros(n, dtype=np.int32)
        res = np.zeros(n, dtype=np.float64)
        if first_check is not None and np.isscalar(tol):
            tol = np.full(n, float(tol))
        fc = None if first_check is None else np.ascontiguousarray(first_check, dtype=np.int32)
        if np.isscalar(tol):
            _check(lib().ats_frame_to_residual(self.h, float(tol), int(check_every), int(max_iterations),
                                               _p(it, ctypes.c_int), _p(res, ctypes.c_double), _stream(stream)))
        else:
            t = np.ascontiguousarray(tol, dtype=np.float64)
            _check(lib().ats_frame_to_residuals(self.h, _p(t, ctypes.c_double), None if fc is None else _p(fc, ctypes.c_int),
                                                int(check_every), int(max_iterations), _p(it, ctypes.c_int),
                                                _p(res, ctypes.c_double), _stream(stream)))
        return it, res

    def energy(self, stream=None):
        out = np.zeros(3, dtype=np.float64)
        _check(lib().ats_energy(self.h, _p(out, ctypes.c_double), _stream(stream)))
        return out

    def residual(self, stream=None):
        out = np.zeros(self.info.num_instances, dtype=np.float64)
        _check(lib().ats_residual(self.h, _p(out, ctypes.c_double), _stream(stream)))
        return out

    def potential(self, stream=None):
        """Per-instance FP64 incremental potential G(x) of the current iterate."""
        out = np.zeros(self.info.num_instances, dtype=np.float64)
        _check(lib().ats_potential(self.h, _p(out, ctypes.c_double), _stream(stream)))
        return out


class MLP:
    """The warm-start network (ats_mlp_*): 24 -> 64 -> 64 -> 64 -> 3, BF16 weights."""

    def __init__(self, seed=0):
        h = _vp()
        _check(lib().ats_mlp_create(int(seed), ctypes.byref(h)))
        self.h = h
        self.nparams = lib().ats_mlp_param_count()

    def close(self):
        if getattr(self, "h", None):
            lib().ats_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        _check(lib().ats_mlp_get_params(self.h, _p(out, ctypes.c_float)))
        return out

    def set_params(self, theta):
        t = np.ascontiguousarray(theta, dtype=np.float32)
        _check(lib().ats_mlp_set_params(self.h, _p(t, ctypes.c_float)))

    def normalization(self):
        out = np.zeros(54, dtype=np.float32)
        _check(lib().ats_mlp_get_normalization(self.h, _p(out, ctypes.c_float)))
        return out

    def set_normalization(self, norm):
        n = np.ascontiguousarray(norm, dtype=np.float32)
        _check(lib().ats_mlp_set_normalization(self.h, _p(n, ctypes.c_float)))

    def fit_normalization(self, dataset, stream=None):
        _check(lib().ats_mlp_fit_normalization(self.h, dataset.h, _stream(stream)))

    def infer(self, features, stream=None):
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros((f.shape[0], 3), dtype=np.float32)
        _check(lib().ats_mlp_infer(self.h, _p(f, ctypes.c_float), f.shape[0], _p(out, ctypes.c_float), _stream(stream)))
        return out

    def gradient(self, features, targets, stream=None):
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float(0.0)
        _check(lib().ats_mlp_gradient(self.h, _p(f, ctypes.c_float), _p(t, ctypes.c_float), f.shape[0],
                                      _p(g, ctypes.c_float), ctypes.byref(loss), _stream(stream)))
        return float(loss.value), g

    def batch_gradient(self, dataset, batch=4096, seed=0, stream=None):
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float(0.0)
        _check(lib().ats_mlp_batch_gradient(self.h, dataset.h, int(batch), int(seed), _p(g, ctypes.c_float),
                                            ctypes.byref(loss), _stream(stream)))
        return float(loss.value), g

    def apply_gradient(self, grad, lr=1e-3, stream=None):
        g = np.ascontiguousarray(grad, dtype=np.float32)
        _check(lib().ats_mlp_apply_gradient(self.h, _p(g, ctypes.c_float), float(lr), _stream(stream)))

    def train(self, dataset, steps, batch=4096, lr=1e-3, seed=0, stream=None):
        loss = ctypes.c_float(0.0)
        _check(lib().ats_mlp_train(self.h, dataset.h, int(steps), int(batch), float(lr), int(seed), ctypes.byref(loss),
                                   _stream(stream)))
        return float(loss.value)


class Dataset:
    """Recorded (features, target) samples on the device (ats_dataset_*)."""

    def __init__(self, capacity):
        h = _vp()
        _check(lib().ats_dataset_create(int(capacity), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().ats_dataset_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        n = ctypes.c_longlong(0)
        _check(lib().ats_dataset_size(self.h, ctypes.byref(n)))
        return int(n.value)

    def read(self, first=0, count=None):
        count = len(self) - first if count is None else count
        f = np.zeros((count, 24), dtype=np.float32)
        t = np.zeros((count, 3), dtype=np.float32)
        _check(lib().ats_dataset_read(self.h, int(first), int(count), _p(f, ctypes.c_float), _p(t, ctypes.c_float)))
        return f, t
