"""Pins the oracle against the reference's own known-answer tests (CPU only).

The reference cannot be compiled here (glm, EnTT, oneTBB, Boost, glibmm and Catch2 are absent),
so its unit tests are restated case by case against the CPU restatement:
  src/NBody/Physics/test/gravity.cpp               pair, quadrupole field and translation cases
  src/NBody/Physics/test/multipoleMomentSummary.cpp quad > oct > hex error ordering
  src/NBody/Physics/test/centerOfMassSummary.cpp    centre-of-mass approximation
  src/NBody/Physics/test/symmetricTensor.cpp        packed index maps and cartesian powers
"""
import itertools

import numpy as np
import pytest

X, Y, Z = 0, 1, 2


# ---- gravity.cpp ----

def test_particle_particle_known_answer(oracle):
    # gravity.cpp:13-26: G = 2, m = 2 at the origin, target at (2, 0, 0) -> a = (-1, 0, 0) within 5e-4
    a = oracle.particle_particle([0, 0, 0], 2.0, [2, 0, 0], G=2.0)
    assert np.linalg.norm(a - np.array([-1.0, 0.0, 0.0])) < 0.0005


def test_quadrupole_field_vector_equals_pair(oracle):
    # gravity.cpp:28-43: the vector part of a particle-node field equals the pair acceleration
    pair = oracle.particle_particle([0, 0, 0], 2.0, [2, 0, 0], G=2.0)
    field = oracle.particle_node(2, [0, 0, 0], 2.0, [2, 0, 0], G=2.0)
    assert np.array_equal(pair, field[:3])


def _offset_case(oracle):
    field = oracle.particle_node(2, [0, 0, 0], 1.0, [2, 0, 0])
    mono = oracle.particle_particle([0, 0, 0], 1.0, [2, 0, 0])
    off = np.array([0.5, 0.0, 0.0], np.float32)
    real = oracle.particle_particle([0, 0, 0], 1.0, np.array([2, 0, 0], np.float32) + off)
    sampled = oracle.field_at(2, field, off)
    return real, sampled, mono


def test_quadrupole_field_accounts_for_offsets(oracle):
    # gravity.cpp:45-83 (first half): evaluating the field at an offset beats the monopole
    real, sampled, mono = _offset_case(oracle)
    assert np.linalg.norm(real - sampled) < np.linalg.norm(real - mono)
    # first-order expansion: -1/4 + (1/4) * 0.5 = -0.125 along x
    assert np.allclose(sampled, [-0.125, 0.0, 0.0], atol=1e-6)


@pytest.mark.xfail(strict=True, reason="gravity.cpp:81-82 asks for < 5 %, but the reference's own "
                   "field expansion (MultipoleAcceleration.h:33-49) gives 21.9 % at offset 0.5; "
                   "the check fails in the reference as well")
def test_quadrupole_field_offset_error_bound(oracle):
    real, sampled, _ = _offset_case(oracle)
    assert np.linalg.norm(real - sampled) / np.linalg.norm(real) < 0.05


@pytest.mark.parametrize("off", list(itertools.product([0.01, 0.1], repeat=3)))
def test_translation_is_reversible_exactly(oracle, off):
    # gravity.cpp:89-117: exact equalities of MultipoleAcceleration::at / translated
    field = oracle.particle_node(2, [0, 0, 0], 2.0, [2, 0, 0], G=2.0)
    off = np.array(off, np.float32)
    moved = oracle.field_translated(2, field, off)
    assert np.array_equal(oracle.field_at(2, field, off), moved[:3])
    assert np.array_equal(field[:3], oracle.field_at(2, moved, -off))
    back = oracle.field_translated(2, moved, -off)
    assert np.array_equal(field[:3], back[:3])


def test_quadrupole_real_scenario(oracle):
    # gravity.cpp:119-153: four bodies, field sampled near the target, error < 5 % and < monopole
    bodies = [([12.237058, 7.9972196, 2.7898774], 0.0570347), ([15.70352, 12.367721, 3.9934757], 0.112188),
              ([12.150897, 13.606152, 3.4104824], 0.371711), ([16.167948, 7.70833, 6.0922756], 0.144094)]
    passive = np.array([0.41169, 1.1282315, 19.398197], np.float32)
    sample = np.array([0.76725245, 1.0069804, 17.802502], np.float32)
    field = np.zeros(oracle.FIELD_SIZE, np.float32)
    actual = np.zeros(3, np.float32)
    for p, m in bodies:
        field = oracle.particle_node(2, p, m, sample, field=field)
        actual = actual + oracle.particle_particle(p, m, passive)
    mono = field[:3]
    approx = oracle.field_at(2, field, passive - sample)
    q = np.linalg.norm(actual - approx) / np.linalg.norm(actual)
    m = np.linalg.norm(actual - mono) / np.linalg.norm(actual)
    assert q < m
    assert q < 0.05


# ---- multipoleMomentSummary.cpp / centerOfMassSummary.cpp ----

def test_multipole_orders_progressively_more_accurate(oracle):
    # multipoleMomentSummary.cpp:12-67
    pm = np.array([[0, 0, -1, 1.0], [0, 0, 1, 1.0], [0, 3, 1, 2.0]], np.float32)
    p = np.array([0, 10, 0], np.float32)
    actual = sum(oracle.particle_particle(b[:3], b[3], p) for b in pm)
    errs = []
    for order in (2, 3, 4):
        _, com_m, moments = oracle.leaf_summary(pm, order)
        errs.append(np.linalg.norm(actual - oracle.node_particle(order, com_m, moments, p)))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] <= 0.005


def test_center_of_mass_accurate_at_distance(oracle):
    # centerOfMassSummary.cpp:12-47
    pm = np.array([[0, 0, -1, 1.0], [0, 0, 1, 1.0]], np.float32)
    p = np.array([0, 20, 0], np.float32)
    actual = sum(oracle.particle_particle(b[:3], b[3], p) for b in pm)
    _, com_m, moments = oracle.leaf_summary(pm, 1)
    approx = oracle.particle_particle(com_m[:3], com_m[3], p)
    assert np.linalg.norm(actual - approx) / np.linalg.norm(actual) < 0.005


# ---- symmetricTensor.cpp ----

def test_order2_member_access(oracle):
    # symmetricTensor.cpp:18-37: packed values 0..5 at XX, XY, XZ, YY, YZ, ZZ (symmetric access)
    expect = {(X, X): 0, (X, Y): 1, (Y, X): 1, (X, Z): 2, (Z, X): 2, (Y, Y): 3, (Y, Z): 4, (Z, Y): 4, (Z, Z): 5}
    for dims, v in expect.items():
        assert oracle.tensor_linear_index(*dims) == v


def test_order3_member_access(oracle):
    # symmetricTensor.cpp:39-60
    expect = {(X, X, X): 0, (X, X, Y): 1, (X, X, Z): 2, (X, Y, Y): 3, (X, Y, Z): 4, (X, Z, Z): 5, (Y, Y, Y): 6,
              (Y, Y, Z): 7, (Y, Z, Z): 8, (Z, Z, Z): 9, (X, Y, X): 1, (Z, Y, X): 4}
    for dims, v in expect.items():
        assert oracle.tensor_linear_index(*dims) == v


def test_linear_to_dimensional_index(oracle):
    # symmetricTensor.cpp:124-137
    assert oracle.tensor_dimensional_index(3, oracle.tensor_linear_index(X, Y, Z)) == (X, Y, Z)
    assert oracle.tensor_dimensional_index(3, oracle.tensor_linear_index(Z, Y, Z)) == (Y, Z, Z)
    assert oracle.tensor_dimensional_index(5, oracle.tensor_linear_index(Z, Y, Z, Y, X)) == (X, Y, Y, Z, Z)


@pytest.mark.parametrize("order", [2, 3, 4, 5])
def test_index_maps_are_inverse(oracle, order):
    for L in range(oracle.UNIQUE[order]):
        assert oracle.tensor_linear_index(*oracle.tensor_dimensional_index(order, L)) == L


def test_cartesian_power(oracle):
    # symmetricTensor.cpp:161-174
    assert np.array_equal(oracle.tensor_cartesian_power(2, [1, 2, 3]), [1, 2, 3, 4, 6, 9])
    assert np.array_equal(oracle.tensor_cartesian_power(3, [1, 2, 3]), [1, 2, 3, 4, 6, 9, 8, 12, 18, 27])


def test_lexicographic_indices(oracle):
    # symmetricTensor.cpp: "Lexicographical Indices" (order 2 enumeration XX, XY, XZ, YX, ...)
    got = [oracle.tensor_lexicographic_index(2, i) for i in range(9)]
    assert got == [(a, b) for a in range(3) for b in range(3)]


def test_matrix_vector_product(oracle):
    # symmetricTensor.cpp "Matrix-vector multiplication": cartesianPower(v) * (1, 0, 0) = v * v.x
    v = np.array([1, 2, 3], np.float32)
    t2 = oracle.tensor_cartesian_power(2, v)
    assert np.array_equal(oracle.tensor2_times_vector(t2, [1, 0, 0]), np.outer(v, v) @ np.array([1, 0, 0]))
    ones = np.ones(6, np.float32)
    assert np.array_equal(oracle.tensor2_times_vector(ones, v), np.ones((3, 3)) @ v)
