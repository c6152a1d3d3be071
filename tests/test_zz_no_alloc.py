"""The allocation-free Morton-code sort (nb_sort_codes_noalloc), through the C ABI on a GPU.

This entry point exists for callers that cannot allocate device memory while they run: an
application whose own pool owns all device memory, or a step loop that must not take
cudaMalloc's implicit device synchronisation. Its scratch lives in one static device array of
at most 2^20 codes, shared by every call and kept between calls, so these tests check that two
calls in a row both agree with the sort inside the force path (nb_update_accelerations +
nb_get_tree), bit for bit as integer work must, and that oversized input is refused.

The file sorts last on purpose, so that a run stopping at its first failure has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_sort(nb, pm):
    """Codes and sort permutation from the existing entry point (the force path's own sort)."""
    with nb.LinearBVHSolver(bodies=pm, rule=nb.Gravity(1.0, 1e-4), theta=0.5, max_leaf_size=16) as s:
        s.update_accelerations()
        t = s.tree()
    codes_in = np.empty_like(t["codes"])
    codes_in[t["ids"]] = t["codes"]  # the unsorted codes, in input order
    return codes_in, t["codes"], t["ids"]


def _noalloc_sort(nb, torch, codes_in):
    n = len(codes_in)
    d_in = torch.from_numpy(codes_in.view(np.int64)).cuda()
    d_sorted = torch.empty(n, dtype=torch.int64, device="cuda")
    d_ids = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = nb.lib().nb_sort_codes_noalloc(d_in.data_ptr(), d_sorted.data_ptr(), d_ids.data_ptr(), n, stream)
    assert rc == 0, rc
    return d_sorted.cpu().numpy().view(np.uint64), d_ids.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_force_path_sort_twice(nb):
    torch = pytest.importorskip("torch")
    cases = [nb.scenarios.plummer(200_000, seed=61)[0], nb.scenarios.uniform_ball(70_001, seed=62)[0]]
    for pm in cases:  # two calls in a row, different sizes: the shared scratch must not leak between them
        codes_in, sorted_ref, ids_ref = _reference_sort(nb, pm)
        got_codes, got_ids = _noalloc_sort(nb, torch, codes_in)
        assert np.array_equal(got_codes, sorted_ref)
        assert np.array_equal(got_ids, ids_ref)


def test_noalloc_sort_repeated_call_same_input(nb):
    torch = pytest.importorskip("torch")
    pm = nb.scenarios.plummer(1 << 20, seed=63)[0]  # the maximum size
    codes_in, sorted_ref, ids_ref = _reference_sort(nb, pm)
    for _ in range(2):
        got_codes, got_ids = _noalloc_sort(nb, torch, codes_in)
        assert np.array_equal(got_codes, sorted_ref)
        assert np.array_equal(got_ids, ids_ref)


def test_noalloc_sort_rejects_oversized_input(nb):
    lib = nb.lib()
    rc = lib.nb_sort_codes_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), (1 << 20) + 1,
                                   None)
    assert rc == -1  # NB_ERR_INVALID_ARGUMENT, refused before any device work
