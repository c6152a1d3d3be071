"""Python binding of the B200 force path (C ABI in include/nbody_gpu.h, library lib/libnbody_b200.so).

The classes mirror the reference's solver interface (src/NBody/Simulation/Solver.h,
src/NBody/Simulation/Solvers/LinearBVHSolver.h, NaiveSolver.h) and its rule
(src/NBody/Physics/Rules/Gravity.h):

    rule = Gravity(G=1.0, epsilon=1e-5)
    solver = QuadrupoleLinearBVHSolver(bodies, rule)   # bodies: (n, 4) x, y, z, m
    solver.theta = 0.5; solver.max_leaf_size = 16      # ActiveTreeSolver::theta, LinearBVH::maxLeafSize
    solver.step()                                      # Solver::step

Every call goes to the compiled library; there is no Python or CPU fallback. Importing this
module raises if the library is missing, and constructing a solver raises if no sm_100 GPU is
usable.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libnbody_b200.so")

NB_OK = 0
# error codes of include/nbody_gpu.h
NB_ERR_INVALID_ARGUMENT = -1
NB_ERR_CUDA = -2
NB_ERR_OUT_OF_MEMORY = -3
NB_ERR_NO_BODIES = -4
NB_ERR_DEVICE_TIMEOUT = -5
NB_ERR_UNSUPPORTED = -6
NB_ERR_DEVICE_CHECK = -7
_STATUS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of device memory",
    -4: "no bodies / nothing computed",
    -5: "device wait limit expired",
    -6: "unsupported",
    -7: "device-side check failed",
}

SOLVER_LINEAR_BVH = 0
SOLVER_NAIVE = 1
SOLVER_DUAL_LINEAR_BVH = 2


class NBodyError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, 'error')} ({status}): {message}")
        self.status = status


class Config(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("order", C.c_int32),
        ("G", C.c_float),
        ("epsilon", C.c_float),
        ("theta", C.c_float),
        ("max_leaf_size", C.c_int32),
        ("time_step", C.c_float),
        ("device", C.c_int32),
    ]


class Counts(C.Structure):
    _fields_ = [
        ("particle_particle", C.c_uint64),
        ("particle_node", C.c_uint64),
        ("node_particle", C.c_uint64),
        ("node_node", C.c_uint64),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("queued", C.c_int64),
        ("running", C.c_int64),
        ("completed", C.c_int64),
        ("body_steps", C.c_int64),
        ("ticks", C.c_int64),
        ("relayouts", C.c_int64),
        ("resident_bytes", C.c_uint64),
        ("cancelled", C.c_int64),
        ("failed_ticks", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PhaseTimes(C.Structure):
    _fields_ = [
        ("bbox_ms", C.c_double),
        ("morton_ms", C.c_double),
        ("sort_ms", C.c_double),
        ("gather_ms", C.c_double),
        ("build_ms", C.c_double),
        ("traverse_ms", C.c_double),
        ("integrate_ms", C.c_double),
        ("passes", C.c_int64),
        ("launches", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# Every symbol include/nbody_gpu.h declares, with its ctypes signature.
_vp, _i32, _i64, _f32p = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_float)
SIGNATURES = {
    "nb_config_default": (None, [C.POINTER(Config)]),
    "nb_create": (C.c_int, [C.POINTER(Config), C.POINTER(_vp)]),
    "nb_destroy": (C.c_int, [_vp]),
    "nb_last_error": (C.c_char_p, [_vp]),
    "nb_solver_id": (C.c_char_p, [_vp]),
    "nb_solver_name": (C.c_char_p, [_vp]),
    "nb_set_config": (C.c_int, [_vp, C.POINTER(Config)]),
    "nb_get_config": (C.c_int, [_vp, C.POINTER(Config)]),
    "nb_set_stream": (C.c_int, [_vp, _vp]),
    "nb_get_stream": (_vp, [_vp]),
    "nb_set_bodies": (C.c_int, [_vp, _i64, _vp, _vp]),
    "nb_set_bodies_device": (C.c_int, [_vp, _i64, _vp, _vp]),
    "nb_body_count": (_i64, [_vp]),
    "nb_get_bodies": (C.c_int, [_vp, _vp, _vp]),
    "nb_get_bodies_device": (C.c_int, [_vp, _vp, _vp]),
    "nb_update_accelerations": (C.c_int, [_vp, _vp]),
    "nb_get_accelerations": (C.c_int, [_vp, _vp]),
    "nb_get_accelerations_device": (C.c_int, [_vp, _vp]),
    "nb_step": (C.c_int, [_vp, _i32]),
    "nb_synchronize": (C.c_int, [_vp]),
    "nb_get_counts": (C.c_int, [_vp, C.POINTER(Counts)]),
    "nb_enable_timing": (C.c_int, [_vp, C.c_int]),
    "nb_get_phase_times": (C.c_int, [_vp, C.POINTER(PhaseTimes)]),
    "nb_get_tree": (C.c_int, [_vp, C.POINTER(_i64), C.POINTER(_i32), _vp, _vp, _vp, _vp]),
    "nb_direct_device": (C.c_int, [_vp, _i64, _vp, _i64, _vp, _vp, _i32]),
    "nb_energy": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nb_sort_codes_noalloc": (C.c_int, [_vp, _vp, _vp, _i64, _vp]),
    "nb_set_instances": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _vp]),
    "nb_instance_count": (_i32, [_vp]),
    "nb_get_instance_roots": (C.c_int, [_vp, _vp]),
    "nb_get_instance_counts": (C.c_int, [_vp, _i32, _vp, _vp]),
    "nb_enable_graphs": (C.c_int, [_vp, C.c_int]),
    "nb_set_fp64_summaries": (C.c_int, [_vp, C.c_int64]),
    "nb_set_traversal_shape": (C.c_int, [_vp, _i32, _i32]),
    "nb_selftest_bounded_wait": (C.c_int, [_i32, _i32]),
    "nb_get_traversal_shape": (C.c_int, [_vp, C.POINTER(_i32), C.POINTER(_i32)]),
    "nb_server_create": (C.c_int, [C.POINTER(Config), C.c_uint64, C.POINTER(_vp)]),
    "nb_server_destroy": (C.c_int, [_vp]),
    "nb_server_last_error": (C.c_char_p, [_vp]),
    "nb_server_context": (_vp, [_vp]),
    "nb_server_submit": (C.c_int, [_vp, _i64, _vp, _vp, C.c_float, _i32, C.POINTER(_i64)]),
    "nb_server_tick": (C.c_int, [_vp, C.POINTER(_i32)]),
    "nb_server_cancel": (C.c_int, [_vp, _i64]),
    "nb_server_inject_alloc_failures": (C.c_int, [_vp, _i32, _i32]),
    "nb_server_status": (C.c_int, [_vp, _i64, C.POINTER(_i32), C.POINTER(_i32)]),
    "nb_server_take_result": (C.c_int, [_vp, _i64, _vp, _vp]),
    "nb_server_get_stats": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "nb_shard_range": (C.c_int, [_i64, _i32, _i32, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "nb_set_shard": (C.c_int, [_vp, _i32, _i32]),
    "nb_shard_buffers": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_i64)]),
    "nb_shard_gathered": (C.c_int, [_vp]),
    "nb_host_alloc": (_vp, [C.c_size_t]),
    "nb_host_free": (None, [_vp]),
}


def build() -> None:
    """Compile the sm_100a library in-tree (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", PKG_ROOT], check=True)


def lib() -> C.CDLL:
    """The loaded library. Raises if it has not been built: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `make -C {PKG_ROOT}`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def shard_range(n: int, rank: int, world: int):
    """(chunk, first, count) of `rank`'s slice of n Morton-ordered bodies (nb_shard_range)."""
    chunk, first, count = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().nb_shard_range(n, rank, world, C.byref(chunk), C.byref(first), C.byref(count))
    if rc != NB_OK:
        raise NBodyError(rc, "invalid shard range")
    return chunk.value, first.value, count.value


class _DeviceArray:
    """A raw device buffer of float4 bodies, exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n, 4), "typestr": "<f4", "data": (ptr, False), "version": 2}


def default_config() -> Config:
    cfg = Config()
    lib().nb_config_default(C.byref(cfg))
    return cfg


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _bodies(a, name="bodies") -> np.ndarray:
    arr = np.ascontiguousarray(a, dtype=np.float32)
    if arr.ndim != 2 or arr.shape[1] != 4:
        raise ValueError(f"{name} must have shape (n, 4)")
    return arr


class Gravity:
    """Gravity(G, epsilon): epsilon is added to r^2 (Gravity.h:195, 207)."""

    def __init__(self, G: float = 1.0, epsilon: float = 0.00001):
        self.G = float(G)
        self.epsilon = float(epsilon)

    def g(self) -> float:
        return self.G


class Solver:
    """A device-resident solver over one set of bodies (Solver<Rule>, Solver.h:26-187)."""

    _solver_kind = SOLVER_LINEAR_BVH
    _order = 1
    _default_theta = 0.3

    def __init__(self, bodies=None, rule: Gravity | None = None, velocities=None, device: int = 0, **kw):
        self._ctx = None
        rule = rule or Gravity()
        cfg = default_config()
        cfg.solver = self._solver_kind
        cfg.order = kw.pop("order", self._order)
        cfg.G = rule.G
        cfg.epsilon = rule.epsilon
        cfg.theta = kw.pop("theta", self._default_theta)
        cfg.max_leaf_size = kw.pop("max_leaf_size", cfg.max_leaf_size)
        cfg.time_step = kw.pop("time_step", cfg.time_step)
        cfg.device = device
        if kw:
            raise TypeError(f"unknown options {sorted(kw)}")
        ctx = C.c_void_p()
        rc = lib().nb_create(C.byref(cfg), C.byref(ctx))
        if rc != NB_OK:
            raise NBodyError(rc, "nb_create failed (no usable sm_100 GPU?)")
        self._ctx = ctx
        self.rule = rule
        if bodies is not None:
            self.set_bodies(bodies, velocities)

    # -- plumbing --
    def _check(self, rc: int):
        if rc != NB_OK:
            raise NBodyError(rc, lib().nb_last_error(self._ctx).decode())

    def close(self):
        if self._ctx is not None:
            lib().nb_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._ctx

    # -- configuration (ActiveTreeSolver::theta, LinearBVH::maxLeafSize, Solver::timeStep) --
    def config(self) -> Config:
        cfg = Config()
        self._check(lib().nb_get_config(self._ctx, C.byref(cfg)))
        return cfg

    def _set(self, **fields):
        cfg = self.config()
        for k, v in fields.items():
            setattr(cfg, k, v)
        self._check(lib().nb_set_config(self._ctx, C.byref(cfg)))

    theta = property(lambda self: self.config().theta, lambda self, v: self._set(theta=v))
    max_leaf_size = property(lambda self: self.config().max_leaf_size, lambda self, v: self._set(max_leaf_size=v))
    time_step = property(lambda self: self.config().time_step, lambda self, v: self._set(time_step=v))
    order = property(lambda self: self.config().order)

    def id(self) -> str:
        return lib().nb_solver_id(self._ctx).decode()

    def name(self) -> str:
        return lib().nb_solver_name(self._ctx).decode()

    def set_stream(self, stream_handle: int | None):
        self._check(lib().nb_set_stream(self._ctx, stream_handle))

    # -- bodies --
    def set_bodies(self, bodies, velocities=None):
        pm = _bodies(bodies)
        vel = None if velocities is None else _bodies(velocities, "velocities")
        if vel is not None and len(vel) != len(pm):
            raise ValueError("velocities and bodies differ in length")
        self._n = len(pm)
        self._check(lib().nb_set_bodies(self._ctx, len(pm), _ptr(pm), None if vel is None else _ptr(vel)))

    def set_bodies_device(self, n: int, d_pos_mass: int, d_vel: int | None = None):
        self._n = n
        self._check(lib().nb_set_bodies_device(self._ctx, n, d_pos_mass, d_vel))

    def set_instances(self, sizes, bodies, velocities=None, thetas=None):
        """Batched independent instances laid out back to back (nb_set_instances)."""
        sizes = np.ascontiguousarray(sizes, np.int64)
        pm = _bodies(bodies)
        if int(sizes.sum()) != len(pm):
            raise ValueError("sizes do not add up to the number of bodies")
        vel = None if velocities is None else _bodies(velocities, "velocities")
        th = None if thetas is None else np.ascontiguousarray(thetas, np.float32)
        self._n = len(pm)
        self._check(lib().nb_set_instances(self._ctx, len(sizes), _ptr(sizes), None if th is None else _ptr(th),
                                           _ptr(pm), None if vel is None else _ptr(vel)))

    def instance_roots(self) -> np.ndarray:
        roots = np.zeros(max(int(lib().nb_instance_count(self._ctx)), 1), np.int32)
        self._check(lib().nb_get_instance_roots(self._ctx, _ptr(roots)))
        return roots

    def instance_count(self) -> int:
        return int(lib().nb_instance_count(self._ctx))

    def instance_counts(self) -> np.ndarray:
        """(particle-particle, node-particle) counts of the last force pass per instance, shape (k, 2)."""
        k = self.instance_count()
        pp = np.zeros(max(k, 1), np.uint64)
        npc = np.zeros(max(k, 1), np.uint64)
        self._check(lib().nb_get_instance_counts(self._ctx, k, _ptr(pp), _ptr(npc)))
        return np.stack([pp[:k], npc[:k]], axis=1)

    def autotune(self, cache=None, candidates=None, passes: int = 3, tolerance: float = 0.0):
        """Pick the leaf size for the current bodies by measurement (see autotune.py)."""
        from . import autotune as at

        return at.autotune(self, cache, candidates or at.DEFAULT_CANDIDATES, passes, tolerance)

    def enable_graphs(self, on: bool = True):
        self._check(lib().nb_enable_graphs(self._ctx, int(on)))

    def set_fp64_summaries(self, min_bodies: int):
        """Combine the summaries of internal nodes with at least `min_bodies` bodies in FP64
        (nb_set_fp64_summaries; 0 turns it off)."""
        self._check(lib().nb_set_fp64_summaries(self._ctx, int(min_bodies)))

    @property
    def traversal_shape(self):
        """(threads per block, partial-accept slab entries) of the traversal launch."""
        t, e = C.c_int32(), C.c_int32()
        self._check(lib().nb_get_traversal_shape(self._ctx, C.byref(t), C.byref(e)))
        return int(t.value), int(e.value)

    @traversal_shape.setter
    def traversal_shape(self, shape):
        self._check(lib().nb_set_traversal_shape(self._ctx, int(shape[0]), int(shape[1])))

    def body_count(self) -> int:
        return int(lib().nb_body_count(self._ctx))

    def bodies(self):
        n = self.body_count()
        pm = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        self._check(lib().nb_get_bodies(self._ctx, _ptr(pm), _ptr(vel)))
        return pm, vel

    # -- Solver::updateAccelerations / Solver::step --
    def update_accelerations(self) -> np.ndarray:
        n = self.body_count()
        acc = np.zeros((n, 4), np.float32)
        self._check(lib().nb_update_accelerations(self._ctx, _ptr(acc)))
        return acc

    def update_accelerations_async(self):
        self._check(lib().nb_update_accelerations(self._ctx, None))

    def accelerations(self) -> np.ndarray:
        acc = np.zeros((self.body_count(), 4), np.float32)
        self._check(lib().nb_get_accelerations(self._ctx, _ptr(acc)))
        return acc

    def step(self, steps: int = 1):
        self._check(lib().nb_step(self._ctx, steps))

    def synchronize(self):
        self._check(lib().nb_synchronize(self._ctx))

    # -- instrumentation and parity taps --
    def counts(self) -> dict:
        c = Counts()
        self._check(lib().nb_get_counts(self._ctx, C.byref(c)))
        return {k: int(getattr(c, k)) for k, _ in Counts._fields_}

    def enable_timing(self, on: bool = True):
        self._check(lib().nb_enable_timing(self._ctx, int(on)))

    def phase_times(self) -> dict:
        t = PhaseTimes()
        self._check(lib().nb_get_phase_times(self._ctx, C.byref(t)))
        return t.as_dict()

    def tree(self) -> dict:
        """Last tree built: sorted codes, sorted caller ids, preorder node records, global bbox."""
        nn = C.c_int64()
        rf = C.c_int32()
        self._check(lib().nb_get_tree(self._ctx, C.byref(nn), C.byref(rf), None, None, None, None))
        n = self.body_count()
        codes = np.zeros(n, np.uint64)
        ids = np.zeros(n, np.uint32)
        recs = np.zeros((max(nn.value, 1), rf.value), np.float32)
        bbox = np.zeros(6, np.float32)
        self._check(lib().nb_get_tree(self._ctx, C.byref(nn), C.byref(rf), _ptr(codes), _ptr(ids), _ptr(recs),
                                      _ptr(bbox)))
        return {"num_nodes": nn.value, "codes": codes, "ids": ids, "records": recs[: nn.value], "bbox": bbox}

    # -- target sharding over ranks (nb_set_shard; see ShardedStepper) --
    def set_shard(self, rank: int, world: int):
        self._check(lib().nb_set_shard(self._ctx, rank, world))

    def shard_buffers(self):
        pos, vel, cap = C.c_void_p(), C.c_void_p(), C.c_int64()
        self._check(lib().nb_shard_buffers(self._ctx, C.byref(pos), C.byref(vel), C.byref(cap)))
        return pos.value, vel.value, cap.value

    def shard_tensors(self, rows: int):
        """torch views (rows, 4) of the current position and velocity buffers (device memory)."""
        import torch

        pos, vel, cap = self.shard_buffers()
        if rows > cap:
            raise ValueError("rows exceed the buffer capacity")
        dev = torch.device("cuda", self.config().device)
        return (torch.as_tensor(_DeviceArray(pos, rows), device=dev),
                torch.as_tensor(_DeviceArray(vel, rows), device=dev))

    def shard_gathered(self):
        self._check(lib().nb_shard_gathered(self._ctx))

    def energy(self):
        """(kinetic, potential) of the current bodies, FP64 on the device (nb_energy)."""
        k, u = C.c_double(), C.c_double()
        self._check(lib().nb_energy(self._ctx, C.byref(k), C.byref(u)))
        return k.value, u.value

    def direct_device(self, n, d_bodies, nt, d_targets, d_acc, precision=32):
        self._check(lib().nb_direct_device(self._ctx, n, d_bodies, nt, d_targets, d_acc, precision))


class LinearBVHSolver(Solver):
    """ActiveTreeSolver<ActiveLinearBVH, DiagonalOverCenterDistance> ("linear-bvh", LinearBVHSolver.h:18-31)."""

    _order = 1


class MultipoleLinearBVHSolver(Solver):
    """MultipoleLinearBVHSolver<Order> (LinearBVHSolver.h:33-44); order 2 is supported on the GPU."""

    _order = 2


class QuadrupoleLinearBVHSolver(MultipoleLinearBVHSolver):
    _order = 2


class NaiveSolver(Solver):
    """NaiveSolver (NaiveSolver.h:12-53): FP32 direct sum over all pairs."""

    _solver_kind = SOLVER_NAIVE


class MultipoleImplicitLinearBVHFMMSolver(Solver):
    """MultipoleImplicitLinearBVHFMMSolver<Order> (ImplicitLinearBVHFMMSolver.h:15-38): dual-tree
    traversal of the linear BVH against itself under DiagonalOverSeparation, with implicit local
    fields of order Order + 1. Order 3 (octupole, "implicit-linear-bvh-fmm-8p") runs on the GPU."""

    _solver_kind = SOLVER_DUAL_LINEAR_BVH
    _order = 3
    _default_theta = 0.5  # ThetaDescentCriterion's default (DescentCriterionType.h:53)


class OctupoleImplicitLinearBVHFMMSolver(MultipoleImplicitLinearBVHFMMSolver):
    _order = 3


class Server:
    """Continuous-batching server of independent simulations (nb_server_*)."""

    QUEUED, RUNNING, DONE = 0, 1, 2

    def __init__(self, rule: Gravity | None = None, order: int = 2, max_leaf_size: int = 16, time_step: float = 1e-3,
                 hbm_budget_bytes: int = 150 * 10 ** 9, device: int = 0):
        rule = rule or Gravity()
        cfg = default_config()
        cfg.order = order
        cfg.G = rule.G
        cfg.epsilon = rule.epsilon
        cfg.max_leaf_size = max_leaf_size
        cfg.time_step = time_step
        cfg.device = device
        h = C.c_void_p()
        rc = lib().nb_server_create(C.byref(cfg), hbm_budget_bytes, C.byref(h))
        if rc != NB_OK:
            raise NBodyError(rc, "nb_server_create failed (no usable sm_100 GPU?)")
        self._h = h

    def _check(self, rc):
        if rc != NB_OK:
            raise NBodyError(rc, lib().nb_server_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().nb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def context(self):
        return lib().nb_server_context(self._h)

    def set_traversal_shape(self, shape):
        """Traversal launch shape (threads per block, tile) of the server's batched passes."""
        self._check(lib().nb_set_traversal_shape(self.context(), int(shape[0]), int(shape[1])))

    def submit(self, bodies, velocities=None, theta: float = 0.5, steps: int = 1) -> int:
        pm = _bodies(bodies)
        vel = None if velocities is None else _bodies(velocities, "velocities")
        rid = C.c_int64()
        self._check(lib().nb_server_submit(self._h, len(pm), _ptr(pm), None if vel is None else _ptr(vel),
                                           float(theta), int(steps), C.byref(rid)))
        return rid.value

    def tick(self) -> int:
        done = C.c_int32()
        self._check(lib().nb_server_tick(self._h, C.byref(done)))
        return done.value

    def status(self, rid: int):
        st, steps = C.c_int32(), C.c_int32()
        self._check(lib().nb_server_status(self._h, rid, C.byref(st), C.byref(steps)))
        return st.value, steps.value

    def take_result(self, rid: int, n: int):
        pm = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        self._check(lib().nb_server_take_result(self._h, rid, _ptr(pm), _ptr(vel)))
        return pm, vel

    def stats(self) -> dict:
        s = ServerStats()
        self._check(lib().nb_server_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def cancel(self, rid: int):
        self._check(lib().nb_server_cancel(self._h, rid))

    def inject_alloc_failures(self, point: int, count: int = 1):
        """Fault injection for tests: the next `count` allocations at `point` fail (0: staging
        buffers of the re-layout, 1: the context's buffers)."""
        self._check(lib().nb_server_inject_alloc_failures(self._h, point, count))


def decode_records(records: np.ndarray, order: int) -> dict:
    """Split exported node records into named fields. Per node: MAC centre and threshold (4 floats),
    link (2 int32: internal = right child's preorder index and -1, leaf = body range), 2 pad floats,
    then the payload: centre of mass and mass, and for order 2 the packed quadrupole."""
    r = np.ascontiguousarray(records, np.float32)
    out = {
        "center": r[:, 0:3],
        "mac_threshold": r[:, 3],
        "link": np.ascontiguousarray(r[:, 4:6]).view(np.int32),
        "com": r[:, 8:11],
        "mass": r[:, 11],
    }
    if order == 2:
        out["quadrupole"] = np.ascontiguousarray(r[:, 12:18])
    return out


def decode_dual_records(records: np.ndarray) -> dict:
    """Split the dual solver's node records (32 floats per node) into named fields: bounding box,
    body count, diagonal length, centre of mass and mass, link (2 int32: leaf = body range,
    internal = right child's preorder index and -1 - first body), quadrupole (6) and octupole (10)
    in the reference's packed layout."""
    r = np.ascontiguousarray(records, np.float32)
    return {
        "bmin": r[:, 0:3],
        "size": np.ascontiguousarray(r[:, 3]).view(np.int32),
        "bmax": r[:, 4:7],
        "diag": r[:, 7],
        "com": r[:, 8:11],
        "mass": r[:, 11],
        "link": np.ascontiguousarray(r[:, 12:14]).view(np.int32),
        "quadrupole": np.ascontiguousarray(r[:, 16:22]),
        "octupole": np.ascontiguousarray(r[:, 22:32]),
    }


from . import scenarios  # noqa: E402
from .sharded import ShardedStepper  # noqa: E402  (host-side scenario generators)
