"""Pins the oracle's polynomial toolkit (a restatement of
crates/protocol/src/domain/fast.rs) to the direct definitions the
reference's own tests compare against: product_oracle, evaluate_oracle and
the diagonal-free Cauchy sum (crates/protocol/src/domain/fast_backend_tests.rs
:41-115), the exact-division cases of :117-141 and :172-190, and the dense
product cases of crates/protocol/src/domain.rs:450-468.  Pure-Python big
integers, small sizes: no GPU.
"""
import random

import pytest

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def fb(xs):
    return b"".join((x % R).to_bytes(32, "little") for x in xs)


def tb(b):
    return [int.from_bytes(b[i:i + 32], "little") for i in range(0, len(b), 32)]


def trim(p):
    p = list(p)
    while len(p) > 1 and p[-1] == 0:
        p.pop()
    return p or [0]


def product_oracle(a, b):  # fast_backend_tests.rs:41-48
    if not a or not b:
        return [0]
    p = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            p[i + j] = (p[i + j] + x * y) % R
    return trim(p)


def evaluate_oracle(poly, x):  # fast_backend_tests.rs:50-54
    v = 0
    for c in reversed(poly):
        v = (v * x + c) % R
    return v


def coefficients(n, offset):  # fast_backend_tests.rs:56-58
    return [offset + i for i in range(n)]


def cauchy_direct(points, weights):
    n = len(points)
    return [sum(weights[j] * pow(points[i] - points[j], R - 2, R) for j in range(n) if j != i) % R
            for i in range(n)]


@pytest.mark.parametrize("ll,rl", [(1, 1), (2, 3), (16, 17), (17, 33), (33, 65)])
def test_products_match_product_oracle(oracle, ll, rl):
    left, right = coefficients(ll, 2), coefficients(rl, 5)
    assert tb(oracle.poly_mul(fb(left), fb(right))) == product_oracle(left, right)


def test_dense_products_with_padding_and_zero_cases(oracle):
    rng = random.Random(3102)
    for ll, rl in [(0, 32), (1, 65), (16, 33), (17, 17), (17, 33), (32, 33), (33, 64), (64, 65), (65, 129)]:
        left = [rng.randrange(R) for _ in range(ll)]
        right = [rng.randrange(R) for _ in range(rl)]
        if left:
            left[-1] = 1
        if right:
            right[-1] = 1
        assert tb(oracle.poly_mul(fb(left), fb(right))) == product_oracle(left, right)
        left, right = left + [0, 0], right + [0, 0, 0]
        assert tb(oracle.poly_mul(fb(left), fb(right))) == product_oracle(left, right)
    assert tb(oracle.poly_mul(fb([0] * 33), fb([1] * 65))) == [0]
    assert tb(oracle.poly_mul(b"", b"")) == [0]
    assert tb(oracle.poly_mul(b"", fb([1]))) == [0]


@pytest.mark.parametrize("size", [0, 1, 2, 3, 7, 17, 33])
def test_tree_matches_direct_definitions(oracle, size):
    points = [5 * (size - i) + 2 for i in range(size)]
    with oracle.Tree(fb(points)) as t:
        van = tb(t.vanishing())
        assert len(van) == size + 1 and van[-1] == 1
        assert all(evaluate_oracle(van, x) == 0 for x in points)
        inv = tb(t.inverse_derivatives())
        for i, x in enumerate(points):
            d = 1
            for j, y in enumerate(points):
                if j != i:
                    d = d * (x - y) % R
            assert inv[i] * d % R == 1
        for degree in (0, size, 2 * size + 3):
            poly = coefficients(degree + 1, 3)
            expected = [evaluate_oracle(poly, x) for x in points]
            assert tb(t.multipoint_eval(fb(poly))) == expected
            f = tb(t.interpolate(fb(expected)))
            assert f == trim(f) and len(f) <= max(1, size)
            assert [evaluate_oracle(f, x) for x in points] == expected
        weights = coefficients(size, 7)
        assert tb(t.cauchy_sums(fb(weights))) == cauchy_direct(points, weights)


def test_tree_rejects_repeated_points(oracle):
    with pytest.raises(ValueError, match="duplicate interpolation point"):
        oracle.Tree(fb([1, 1]))


def test_exact_division_cases(oracle):
    den = [-2 % R, 3, 1]
    quo = [5, 7, 11, 13]
    assert tb(oracle.poly_div_exact(fb(product_oracle(den, quo)), fb(den))) == quo
    for dl, ql in [(1, 1), (1, 17), (3, 19), (17, 3), (19, 35)]:
        den, quo = coefficients(dl, 2), coefficients(ql, 7)
        num = product_oracle(den, quo)
        assert tb(oracle.poly_div_exact(fb(num), fb(den))) == quo
        if dl > 1:
            num[0] += 1
            with pytest.raises(ValueError, match="nonzero remainder"):
                oracle.poly_div_exact(fb(num), fb(den))
    with pytest.raises(ValueError, match="zero polynomial"):
        oracle.poly_div_exact(fb([1]), b"")
    with pytest.raises(ValueError, match="nonzero remainder"):
        oracle.poly_div_exact(fb([1]), fb([0, 1]))
    assert tb(oracle.poly_div_exact(b"", fb([1]))) == [0]
