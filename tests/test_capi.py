"""The C-ABI library (CPU-side checks): it loads, exports every symbol include/nbody_gpu.h declares,
and refuses to run without a usable GPU instead of falling back to a CPU path."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "nbody_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("nb_create", "nb_destroy", "nb_set_bodies", "nb_update_accelerations", "nb_step",
                     "nb_get_tree", "nb_get_counts", "nb_direct_device"):
        assert required in names


def test_library_exports_every_declared_symbol(nb):
    lib = ctypes.CDLL(nb.LIB_PATH)
    missing = [name for name in declared_functions() if not hasattr(lib, name)]
    assert not missing, f"symbols declared in nbody_gpu.h but not exported: {missing}"


def test_binding_covers_every_declared_symbol(nb):
    assert set(declared_functions()) <= set(nb.SIGNATURES)


def test_default_config_matches_reference_defaults(nb):
    cfg = nb.default_config()
    assert cfg.G == 1.0
    assert abs(cfg.epsilon - 1e-5) < 1e-12   # Gravity.h:195
    assert abs(cfg.theta - 0.3) < 1e-7       # ActiveTreeSolver.h:21
    assert cfg.max_leaf_size == 64           # LinearBVH.h:88
    assert abs(cfg.time_step - 0.001) < 1e-9  # Solver.h:34
    assert cfg.order == 1


def test_library_build_targets_sm100a():
    so = os.path.join(REPO, "n-body_b200", "lib", "libnbody_b200.so")
    assert os.path.exists(so)
    mk = open(os.path.join(REPO, "n-body_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_no_gpu_fails_loudly(nb):
    """Without a CUDA device the solver must raise, never compute on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(nb.NBodyError):
        nb.LinearBVHSolver()


def test_invalid_config_rejected_before_device(nb):
    cfg = nb.default_config()
    cfg.order = 7
    ctx = ctypes.c_void_p()
    assert nb.lib().nb_create(ctypes.byref(cfg), ctypes.byref(ctx)) == -6
    cfg.order = 1
    cfg.max_leaf_size = 0
    assert nb.lib().nb_create(ctypes.byref(cfg), ctypes.byref(ctx)) == -1
