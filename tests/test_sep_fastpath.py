"""The float fast path of the dual tree's separation test decides exactly as the double path.

`sep_test` in `n-body_b200/csrc/dualtree.cu` decides sep >= B, where sep is the reference's
separation (DiagonalOverSeparation.h:29-49): the rounded lengths lu = RN(sqrt(su)) and
lv = RN(sqrt(sv)) of the two separation vectors, combined as RN_float(sqrt(lu^2 + lv^2)) in double.
When both vectors are nonzero it first compares q = RN(su + sv) with RN(B^2) (1 +- 2^-18) and
takes the double path only in between. This restates both paths in numpy (IEEE float32 and
float64 arithmetic, as on the device) and checks, on random inputs and on inputs built to lie
within a few ulps of the threshold, that every case the fast path decides is decided as the
double path decides it.
"""
import numpy as np

F32 = np.float32


def exact(su, sv, B):
    lu = np.sqrt(su).astype(np.float64)
    lv = np.sqrt(sv).astype(np.float64)
    sep = np.sqrt(lu * lu + lv * lv).astype(np.float32)
    return sep >= B


def fast(su, sv, B):
    """(decided, value): the fast path's verdict where it decides."""
    b2 = (B * B).astype(np.float32)
    q = (su + sv).astype(np.float32)
    ok = (b2 >= F32(1e-30)) & (b2 <= F32(1e30))
    hi = (b2 * F32(1.0 + 2.0 ** -18)).astype(np.float32)
    lo = (b2 * F32(1.0 - 2.0 ** -18)).astype(np.float32)
    yes = ok & (q >= hi)
    no = ok & (q < lo)
    return yes | no, yes


def check(su, sv, B):
    su, sv, B = su.astype(np.float32), sv.astype(np.float32), B.astype(np.float32)
    keep = (su > 0) & (sv > 0) & np.isfinite(su) & np.isfinite(sv) & (B > 0) & np.isfinite(B)
    su, sv, B = su[keep], sv[keep], B[keep]
    with np.errstate(over="ignore", invalid="ignore"):
        decided, value = fast(su, sv, B)
        ref = exact(su, sv, B)
    assert np.array_equal(value[decided], ref[decided])
    return decided.mean()


def test_random_inputs():
    rng = np.random.default_rng(11)
    n = 2_000_000
    su = 10.0 ** rng.uniform(-14, 14, n)
    sv = su * 10.0 ** rng.uniform(-6, 6, n)
    B = np.sqrt(su + sv) * rng.uniform(0.0, 3.0, n)
    frac = check(su, sv, B)
    assert frac > 0.99  # the double path is the rare case


def test_near_threshold_inputs():
    rng = np.random.default_rng(12)
    n = 2_000_000
    su = (10.0 ** rng.uniform(-12, 12, n)).astype(np.float32)
    sv = (su * 10.0 ** rng.uniform(-3, 3, n)).astype(np.float32)
    lu = np.sqrt(su).astype(np.float64)
    lv = np.sqrt(sv).astype(np.float64)
    sep = np.sqrt(lu * lu + lv * lv)
    # B within a relative 1e-5 of the separation, then moved by up to 4 ulps either way
    B = (sep * (1.0 + rng.uniform(-1e-5, 1e-5, n))).astype(np.float32)
    B = (B.view(np.int32) + rng.integers(-4, 5, n).astype(np.int32)).view(np.float32)
    check(su, sv, B)
