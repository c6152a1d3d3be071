"""Oracle bindings (test infrastructure only).

ctypes wrappers over ``oracle/_build/libnbody_oracle.so``, the FP32 CPU restatement of the
reference's Barnes-Hut force path (see nbody_oracle.cpp for the file:line of every restated
piece). Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, and only as the checker or as the timed CPU baseline; the product path never does.

Arrays of bodies are float32 with 4 values per body: x, y, z, mass (velocities: vx, vy, vz, 0).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libnbody_oracle.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")

_lib = None


def build() -> None:
    """Compile the oracle library with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


NATIVE_PATH = os.path.join(HERE, "_build", "libnbody_oracle_native.so")
NATIVE_STAMP = NATIVE_PATH + ".host"
_timing_lib = None


def _host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def timing_lib() -> C.CDLL:
    """The timing build (-O3 -march=native) for the CPU baseline, compiled on first use for the
    host it runs on (rebuilt when the host's CPU model differs from the one it was built for)."""
    global _timing_lib
    if _timing_lib is None:
        cpu = _host_cpu()
        stamp = open(NATIVE_STAMP).read() if os.path.exists(NATIVE_STAMP) else None
        if stamp != cpu or not os.path.exists(NATIVE_PATH):
            if os.path.exists(NATIVE_PATH):
                os.remove(NATIVE_PATH)
            subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
            with open(NATIVE_STAMP, "w") as f:
                f.write(cpu)
        _timing_lib = _load(NATIVE_PATH)
    return _timing_lib


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _load(LIB_PATH)
    return _lib


def _load(path: str) -> C.CDLL:
    """The library at `path` with every exported function's ctypes signature."""
    L = C.CDLL(path)
    i64, i32, f32, f64 = C.c_int64, C.c_int32, C.c_float, C.c_double
    sig = {
        "or_bbox": (None, [i64, _f32p, _f32p]),
        "or_morton": (None, [i64, _f32p, _f32p, _u64p]),
        "or_sort": (None, [i64, _u64p, _u32p]),
        "or_build": (i64, [i64, _u64p, i32, _i32p, _i32p, _i32p, _i32p]),
        "or_summarize": (C.c_int, [i64, _i32p, _i32p, _i32p, _i32p, _f32p, i32, _f32p, _f32p, _f32p]),
        "or_bh_accelerations": (i64, [i64, _f32p, f32, f32, f32, i32, i32, _f32p, _u64p, i32]),
        "or_bh_targets": (i64, [i64, _f32p, i64, _f32p, f32, f32, f32, i32, i32, _f32p, _u64p, i32]),
        "or_direct_f32": (None, [i64, _f32p, i64, C.c_void_p, f32, f32, _f32p, i32]),
        "or_direct_f64": (None, [i64, _f32p, i64, C.c_void_p, f64, f64, _f64p, i32]),
        "or_kick_drift": (None, [i64, _f32p, _f32p, _f32p, f32]),
        "or_max_threads": (i32, []),
        "or_particle_particle": (None, [f32, f32, _f32p, f32, _f32p, _f32p]),
        "or_leaf_summary": (C.c_int, [i64, _f32p, i32, _f32p, _f32p, _f32p]),
        "or_node_particle": (C.c_int, [i32, f32, f32, _f32p, _f32p, _f32p, _f32p]),
        "or_particle_node": (C.c_int, [i32, f32, f32, _f32p, f32, _f32p, _f32p]),
        "or_field_at": (C.c_int, [i32, _f32p, _f32p, _f32p]),
        "or_field_translated": (C.c_int, [i32, _f32p, _f32p, _f32p]),
        "or_dual_accelerations": (i64, [i64, _f32p, f32, f32, f32, i32, i32, _f32p, _u64p, i32]),
        "or_tensor_linear_index": (i32, [i32, _i32p]),
        "or_tensor_dimensional_index": (C.c_int, [i32, i32, _i32p]),
        "or_tensor_lexicographic_index": (C.c_int, [i32, i32, _i32p]),
        "or_tensor_cartesian_power": (C.c_int, [i32, _f32p, _f32p]),
        "or_tensor2_times_vector": (None, [_f32p, _f32p, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def _bodies(pm) -> np.ndarray:
    a = np.ascontiguousarray(pm, dtype=np.float32)
    assert a.ndim == 2 and a.shape[1] == 4
    return a


def bbox(pm) -> np.ndarray:
    pm = _bodies(pm)
    out = np.zeros(6, np.float32)
    lib().or_bbox(len(pm), pm, out)
    return out


def morton_codes(pm, box=None) -> np.ndarray:
    pm = _bodies(pm)
    box = bbox(pm) if box is None else np.ascontiguousarray(box, np.float32)
    codes = np.zeros(len(pm), np.uint64)
    lib().or_morton(len(pm), pm, box, codes)
    return codes


def sort_codes(codes) -> np.ndarray:
    codes = np.ascontiguousarray(codes, np.uint64)
    perm = np.zeros(len(codes), np.uint32)
    lib().or_sort(len(codes), codes, perm)
    return perm


def build_tree(sorted_codes, leaf: int):
    """Preorder LinearBVH topology: (begin, end, left, right); left = right = -1 at leaves."""
    sc = np.ascontiguousarray(sorted_codes, np.uint64)
    n = len(sc)
    cap = max(2 * n, 1)
    b, e, l, r = (np.zeros(cap, np.int32) for _ in range(4))
    nn = lib().or_build(n, sc, leaf, b, e, l, r)
    return b[:nn].copy(), e[:nn].copy(), l[:nn].copy(), r[:nn].copy()


def summarize(tree, pm_sorted, order: int):
    """Per-node (bbox[6], com_m[4], moments[31]) exactly as the reference's summaries."""
    b, e, l, r = (np.ascontiguousarray(x, np.int32) for x in tree)
    nn = len(b)
    pm_sorted = _bodies(pm_sorted)
    bb = np.zeros((max(nn, 1), 6), np.float32)
    cm = np.zeros((max(nn, 1), 4), np.float32)
    mo = np.zeros((max(nn, 1), 31), np.float32)
    rc = lib().or_summarize(nn, b, e, l, r, pm_sorted, order, bb, cm, mo)
    assert rc == 0
    return bb[:nn], cm[:nn], mo[:nn]


def bh_accelerations(pm, G=1.0, eps=1e-5, theta=0.5, leaf=16, order=1, threads=0, L=None):
    """ActiveTreeSolver (LinearBVH, DiagonalOverCenterDistance, Gravity) accelerations in input
    order, and the (particle-particle, node-particle) interaction counts. L: the library to run
    (default: the parity build; timing_lib() for the CPU baseline)."""
    pm = _bodies(pm)
    acc = np.zeros((len(pm), 4), np.float32)
    counts = np.zeros(2, np.uint64)
    nn = (L or lib()).or_bh_accelerations(len(pm), pm, G, eps, theta, leaf, order, acc, counts, threads)
    assert nn >= 0
    return acc, counts


def bh_targets(pm, targets, G=1.0, eps=1e-5, theta=0.5, leaf=16, order=1, threads=0):
    pm = _bodies(pm)
    targets = _bodies(targets)
    acc = np.zeros((len(targets), 4), np.float32)
    counts = np.zeros(2, np.uint64)
    nn = lib().or_bh_targets(len(pm), pm, len(targets), targets, G, eps, theta, leaf, order, acc, counts, threads)
    assert nn >= 0
    return acc, counts


def dual_accelerations(pm, G=1.0, eps=1e-5, theta=0.4, leaf=64, order=3, threads=0):
    """MultipoleImplicitLinearBVHFMMSolver<order> (dual-tree, implicit local field of order+1):
    accelerations in input order and the (pp, np, pn, nn) interaction counts."""
    pm = _bodies(pm)
    acc = np.zeros((len(pm), 4), np.float32)
    counts = np.zeros(4, np.uint64)
    nn = lib().or_dual_accelerations(len(pm), pm, G, eps, theta, leaf, order, acc, counts, threads)
    assert nn >= 0
    return acc, counts


def direct_f32(pm, idx=None, G=1.0, eps=1e-5, threads=0) -> np.ndarray:
    pm = _bodies(pm)
    if idx is None:
        nt, ptr, keep = len(pm), None, None
    else:
        keep = np.ascontiguousarray(idx, np.int64)
        nt, ptr = len(keep), keep.ctypes.data
    acc = np.zeros((nt, 4), np.float32)
    lib().or_direct_f32(len(pm), pm, nt, ptr, G, eps, acc, threads)
    return acc


def direct_f64(pm, idx=None, G=1.0, eps=1e-5, threads=0) -> np.ndarray:
    pm = _bodies(pm)
    if idx is None:
        nt, ptr, keep = len(pm), None, None
    else:
        keep = np.ascontiguousarray(idx, np.int64)
        nt, ptr = len(keep), keep.ctypes.data
    acc = np.zeros((nt, 3), np.float64)
    lib().or_direct_f64(len(pm), pm, nt, ptr, G, eps, acc, threads)
    return acc


def kick_drift(pm, vel, acc, dt: float, L=None):
    pm = _bodies(pm).copy()
    vel = _bodies(vel).copy()
    acc = _bodies(acc)
    (L or lib()).or_kick_drift(len(pm), pm, vel, acc, dt)
    return pm, vel


def max_threads(L=None) -> int:
    return int((L or lib()).or_max_threads())


# ---- rule-level helpers ----

def particle_particle(active, m, passive, G=1.0, eps=1e-5) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().or_particle_particle(G, eps, np.asarray(active, np.float32), m, np.asarray(passive, np.float32), out)
    return out


def leaf_summary(pm, order: int):
    pm = _bodies(pm)
    bb, cm, mo = np.zeros(6, np.float32), np.zeros(4, np.float32), np.zeros(31, np.float32)
    assert lib().or_leaf_summary(len(pm), pm, order, bb, cm, mo) == 0
    return bb, cm, mo


def node_particle(order, com_m, moments, passive, G=1.0, eps=1e-5) -> np.ndarray:
    out = np.zeros(3, np.float32)
    rc = lib().or_node_particle(order, G, eps, np.asarray(com_m, np.float32), np.asarray(moments, np.float32),
                                np.asarray(passive, np.float32), out)
    assert rc == 0
    return out


FIELD_SIZE = 55  # vector(3) + t2(6) + t3(10) + t4(15) + t5(21)


def particle_node(order, active, m, center, field=None, G=1.0, eps=1e-5) -> np.ndarray:
    f = np.zeros(FIELD_SIZE, np.float32) if field is None else np.array(field, np.float32)
    rc = lib().or_particle_node(order, G, eps, np.asarray(active, np.float32), m, np.asarray(center, np.float32), f)
    assert rc == 0
    return f


def field_at(order, field, off) -> np.ndarray:
    out = np.zeros(3, np.float32)
    assert lib().or_field_at(order, np.asarray(field, np.float32), np.asarray(off, np.float32), out) == 0
    return out


def field_translated(order, field, off) -> np.ndarray:
    out = np.zeros(FIELD_SIZE, np.float32)
    assert lib().or_field_translated(order, np.asarray(field, np.float32), np.asarray(off, np.float32), out) == 0
    return out


# ---- symmetric tensor helpers (index maps of SymmetricTensor3) ----
X, Y, Z = 0, 1, 2
UNIQUE = {1: 3, 2: 6, 3: 10, 4: 15, 5: 21}


def tensor_linear_index(*dims) -> int:
    d = np.asarray(dims, np.int32)
    return int(lib().or_tensor_linear_index(len(d), d))


def tensor_dimensional_index(order: int, L: int) -> tuple:
    d = np.zeros(order, np.int32)
    assert lib().or_tensor_dimensional_index(order, L, d) == 0
    return tuple(int(x) for x in d)


def tensor_lexicographic_index(order: int, I: int) -> tuple:
    d = np.zeros(order, np.int32)
    assert lib().or_tensor_lexicographic_index(order, I, d) == 0
    return tuple(int(x) for x in d)


def tensor_cartesian_power(order: int, v) -> np.ndarray:
    out = np.zeros(UNIQUE[order], np.float32)
    assert lib().or_tensor_cartesian_power(order, np.asarray(v, np.float32), out) == 0
    return out


def tensor2_times_vector(t2, v) -> np.ndarray:
    out = np.zeros(3, np.float32)
    lib().or_tensor2_times_vector(np.asarray(t2, np.float32), np.asarray(v, np.float32), out)
    return out
