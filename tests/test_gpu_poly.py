"""Device polynomial toolkit parity (dvgpu_bn254_poly_* / dvgpu_bn254_tree_*).

Each entry point is compared with the oracle's restatement of
crates/protocol/src/domain/fast.rs on the same inputs -- the cases of the
reference's fast_backend_tests.rs (:60-115, :117-141, :172-190) and
domain.rs:450-468, then seeded uniform inputs -- and at larger sizes through
size-independent properties (interpolate then evaluate gives the values
back, the vanishing polynomial is zero at every point, (a b) / b = a).
"""
import random

import pytest

pytestmark = pytest.mark.gpu

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def fb(xs):
    return b"".join((x % R).to_bytes(32, "little") for x in xs)


def tb(b):
    return [int.from_bytes(b[i:i + 32], "little") for i in range(0, len(b), 32)]


def coefficients(n, offset):
    return [offset + i for i in range(n)]


def test_products_match_oracle(backend, oracle, dv):
    for ll, rl in [(1, 1), (2, 3), (16, 17), (17, 33), (33, 65)]:
        a, b = fb(coefficients(ll, 2)), fb(coefficients(rl, 5))
        assert backend.poly_multiply(a, b) == oracle.poly_mul(a, b)
    rng = random.Random(3102)
    for ll, rl in [(0, 32), (1, 65), (16, 33), (17, 17), (32, 33), (65, 129), (129, 130), (1000, 3000)]:
        a = [rng.randrange(R) for _ in range(ll)]
        b = [rng.randrange(R) for _ in range(rl)]
        for pad in (0, 3):
            x, y = fb(a + [0] * pad), fb(b + [0] * pad)
            assert backend.poly_multiply(x, y) == oracle.poly_mul(x, y)
    assert tb(backend.poly_multiply(fb([0] * 33), fb([1] * 65))) == [0]
    assert tb(backend.poly_multiply(b"", b"")) == [0]
    assert tb(backend.poly_multiply(fb([1, 1]), fb([1, 1]))) == [1, 2, 1]


def test_large_product_matches_oracle(backend, oracle):
    a, b = oracle.uniform_fr(41, 1 << 15), oracle.uniform_fr(42, (1 << 15) + 7)
    assert backend.poly_multiply(a, b) == oracle.poly_mul(a, b)


def test_exact_division_matches_oracle(backend, oracle, dv):
    den = fb([-2 % R, 3, 1])
    num = oracle.poly_mul(den, fb([5, 7, 11, 13]))
    assert tb(backend.poly_divide_exact(num, den)) == [5, 7, 11, 13]
    for dl, ql in [(1, 1), (1, 17), (3, 19), (17, 3), (19, 35), (300, 4000)]:
        den, quo = fb(coefficients(dl, 2)), fb(coefficients(ql, 7))
        num = oracle.poly_mul(den, quo)
        assert backend.poly_divide_exact(num, den) == quo
        assert backend.poly_divide_exact(num + fb([0, 0]), den + fb([0])) == quo  # untrimmed operands
        if dl > 1:
            bad = fb([tb(num[:32])[0] + 1]) + num[32:]
            with pytest.raises(dv.DvgpuError) as e:
                backend.poly_divide_exact(bad, den)
            assert e.value.status == -1 and "nonzero remainder" in e.value.message
    # uniform operands: the vanishing polynomial of a sparse update divides its numerator
    q, d = oracle.uniform_fr(43, 2049), oracle.uniform_fr(44, 1025)
    assert backend.poly_divide_exact(oracle.poly_mul(q, d), d) == q
    with pytest.raises(dv.DvgpuError, match="zero polynomial"):
        backend.poly_divide_exact(fb([1]), b"")
    with pytest.raises(dv.DvgpuError, match="zero polynomial"):
        backend.poly_divide_exact(fb([1]), fb([0, 0]))
    with pytest.raises(dv.DvgpuError, match="nonzero remainder"):
        backend.poly_divide_exact(fb([1]), fb([0, 1]))
    assert tb(backend.poly_divide_exact(b"", fb([1]))) == [0]
    assert tb(backend.poly_divide_exact(fb([0, 0]), fb([3, 1]))) == [0]


def test_division_skips_a_coset_that_meets_a_root(backend, oracle):
    # X - 5 vanishes at the first coset's point 5 w^0: the next shift must be taken.
    den = fb([R - 5, 1])
    quo = oracle.uniform_fr(45, 63)
    assert backend.poly_divide_exact(oracle.poly_mul(quo, den), den) == quo


def _check_tree(backend, oracle, points, degrees, seed):
    n = len(points) // 32
    with backend.tree_create(points) as t, oracle.Tree(points) as o:
        assert t.vanishing() == o.vanishing()
        assert t.inverse_derivatives() == o.inverse_derivatives()
        for k, degree in enumerate(degrees):
            poly = oracle.uniform_fr(seed + k, degree + 1)
            values = t.multipoint_eval(poly)
            assert values == o.multipoint_eval(poly)
            assert t.interpolate(values) == o.interpolate(values)
        weights = oracle.uniform_fr(seed + 99, n)
        assert t.cauchy_sums(weights) == o.cauchy_sums(weights)
        assert t.interpolate(weights) == o.interpolate(weights)


@pytest.mark.parametrize("size", [0, 1, 2, 3, 7, 17, 33])
def test_tree_reference_cases(backend, oracle, size):
    points = fb([5 * (size - i) + 2 for i in range(size)])
    with backend.tree_create(points) as t, oracle.Tree(points) as o:
        assert t.vanishing() == o.vanishing()
        assert t.inverse_derivatives() == o.inverse_derivatives()
        for degree in (0, size, 2 * size + 3):
            poly = fb(coefficients(degree + 1, 3))
            assert t.multipoint_eval(poly) == o.multipoint_eval(poly)
            values = o.multipoint_eval(poly)
            assert t.interpolate(values) == o.interpolate(values)
        weights = fb(coefficients(size, 7))
        assert t.cauchy_sums(weights) == o.cauchy_sums(weights)


@pytest.mark.parametrize("size", [64, 255, 256, 257, 1000])
def test_tree_uniform_points_match_oracle(backend, oracle, size):
    _check_tree(backend, oracle, oracle.uniform_fr(700 + size, size), [0, size - 1, size, 3 * size + 5], 800)


def test_tree_rows_match_single_calls(backend, oracle):
    n, rows = 300, 5
    points = oracle.uniform_fr(901, n)
    with backend.tree_create(points) as t:
        polys = [oracle.uniform_fr(910 + r, 2 * n) for r in range(rows)]
        vals = t.multipoint_eval(b"".join(polys), rows)
        assert vals == b"".join(t.multipoint_eval(p) for p in polys)
        values = [oracle.uniform_fr(920 + r, n) for r in range(rows)]
        values[2] = fb([0] * n)           # the zero polynomial: [0]
        values[3] = fb([7] * n)           # a constant: trimmed to one coefficient
        many = t.interpolate(b"".join(values), rows)
        assert many == [t.interpolate(v) for v in values]
        assert tb(many[2]) == [0] and tb(many[3]) == [7]
        sums = t.cauchy_sums(b"".join(values), rows)
        assert sums == b"".join(t.cauchy_sums(v) for v in values)


def test_tree_large_properties(backend, oracle):
    n = 4096  # the power-of-two case: A mod X^N - 1 wraps the leading term
    points = oracle.uniform_fr(930, n)
    values = oracle.uniform_fr(931, n)
    with backend.tree_create(points) as t:
        van = t.vanishing()
        assert len(van) == 32 * (n + 1) and tb(van[-32:]) == [1]
        assert t.multipoint_eval(van) == fb([0] * n)
        f = t.interpolate(values)
        assert len(f) <= 32 * n
        assert t.multipoint_eval(f) == values
        with oracle.Tree(points[:32 * 512]) as o, backend.tree_create(points[:32 * 512]) as small:
            assert small.cauchy_sums(values[:32 * 512]) == o.cauchy_sums(values[:32 * 512])


def test_tree_errors(backend, dv):
    with pytest.raises(dv.DvgpuError) as e:
        backend.tree_create(fb([1, 2, 3, 2]))
    assert e.value.status == -1 and "duplicate interpolation point" in e.value.message
    with pytest.raises(dv.DvgpuError, match="non-canonical"):
        backend.tree_create(R.to_bytes(32, "little"))
    with backend.tree_create(fb([1, 2, 3])) as t:
        with pytest.raises(dv.DvgpuError, match="interpolation value count differs"):
            t.interpolate(fb([1, 2]))
        with pytest.raises(dv.DvgpuError, match="Cauchy weight count differs"):
            t.cauchy_sums(fb([1, 2, 3, 4]))
        with pytest.raises(dv.DvgpuError, match="interpolation value count differs"):
            t.interpolate(b"")
        assert t.multipoint_eval(b"") == fb([0, 0, 0])
    # the owner stays usable after argument errors
    assert tb(backend.poly_multiply(fb([2]), fb([3]))) == [6]
