"""ctypes view of the BN254 CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py as the checker.  The CUDA library never imports this module.
All byte layouts are the reference's canonical wire formats
(crates/gpu/src/codec.rs:25-111, crates/gpu/src/resident.rs:419-431):
Fr/Fq 32-byte little-endian canonical, G1 64 bytes x||y, G2 128 bytes
x.c0||x.c1||y.c0||y.c1, infinity all zero.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u8p = ctypes.c_char_p
        sz = ctypes.c_size_t
        L.oracle_msm_g1.argtypes = [u8p, u8p, sz, u8p, ctypes.c_int, ctypes.c_int]
        L.oracle_msm_g2.argtypes = [u8p, u8p, sz, u8p, ctypes.c_int, ctypes.c_int]
        L.oracle_sparse_msm_g1.argtypes = [u8p, sz, ctypes.c_void_p, u8p, sz, u8p, ctypes.c_int]
        L.oracle_ntt.argtypes = [u8p, sz, ctypes.c_int]
        L.oracle_g1_fft.argtypes = [u8p, sz, sz, ctypes.c_int, u8p, ctypes.c_int]
        L.oracle_g1_scale.argtypes = [u8p, u8p, sz, u8p, ctypes.c_int]
        L.oracle_fixed_base_g1.argtypes = [u8p, sz, u8p, ctypes.c_int]
        L.oracle_fixed_base_g2.argtypes = [u8p, sz, u8p, ctypes.c_int]
        L.oracle_g2_check.argtypes = [u8p, sz, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int]
        L.oracle_g1_on_curve.argtypes = [u8p]
        L.oracle_g2_on_curve.argtypes = [u8p]
        L.oracle_chacha_uniform.argtypes = [ctypes.c_uint64, sz, ctypes.c_int, u8p]
        L.oracle_fr_powers.argtypes = [u8p, sz, u8p]
        L.oracle_g2_twist_points.argtypes = [ctypes.c_uint64, sz, u8p]
        L.oracle_g2_twist_points.restype = sz
        L.oracle_g1_add.argtypes = [u8p, u8p, u8p]
        L.oracle_g2_add.argtypes = [u8p, u8p, u8p]
        L.oracle_g2_mul_r.argtypes = [u8p, u8p]
        L.oracle_poly_mul.argtypes = [u8p, sz, u8p, sz, u8p]
        L.oracle_poly_mul.restype = sz
        L.oracle_poly_div_exact.argtypes = [u8p, sz, u8p, sz, u8p, ctypes.POINTER(sz)]
        L.oracle_tree_new.argtypes = [u8p, sz]
        L.oracle_tree_new.restype = ctypes.c_void_p
        L.oracle_tree_free.argtypes = [ctypes.c_void_p]
        L.oracle_tree_vanishing.argtypes = [ctypes.c_void_p, u8p]
        L.oracle_tree_vanishing.restype = sz
        L.oracle_tree_inverse_derivatives.argtypes = [ctypes.c_void_p, u8p]
        L.oracle_tree_eval.argtypes = [ctypes.c_void_p, u8p, sz, u8p]
        L.oracle_tree_interpolate.argtypes = [ctypes.c_void_p, u8p, u8p]
        L.oracle_tree_interpolate.restype = sz
        L.oracle_tree_cauchy.argtypes = [ctypes.c_void_p, u8p, u8p]
        L.oracle_pairing.argtypes = [u8p, u8p, sz, u8p, ctypes.c_int]
        L.oracle_pairing_check.argtypes = [u8p, u8p, ctypes.c_void_p, sz, u8p, ctypes.c_int]
        _lib = L
    return _lib


def _buf(n):
    return ctypes.create_string_buffer(n)


def msm_g1(points: bytes, scalars: bytes, threads=0, naive=False) -> bytes:
    n = len(scalars) // 32
    assert len(points) == 64 * n
    out = _buf(64)
    if lib().oracle_msm_g1(points, scalars, n, out, threads, int(naive)) != 0:
        raise ValueError("oracle: non-canonical G1 input")
    return out.raw


def msm_g2(points: bytes, scalars: bytes, threads=0, naive=False) -> bytes:
    n = len(scalars) // 32
    assert len(points) == 128 * n
    out = _buf(128)
    if lib().oracle_msm_g2(points, scalars, n, out, threads, int(naive)) != 0:
        raise ValueError("oracle: non-canonical G2 input")
    return out.raw


def sparse_msm_g1(bases: bytes, indices, values: bytes, threads=0) -> bytes:
    idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
    out = _buf(64)
    rc = lib().oracle_sparse_msm_g1(bases, len(bases) // 64, idx.ctypes.data, values, len(idx), out, threads)
    if rc != 0:
        raise ValueError("oracle: sparse index out of range")
    return out.raw


NTT_KINDS = {"forward": 0, "inverse": 1, "coset_forward": 2, "coset_inverse": 3}


def g1_fft(points: bytes, n: int, inverse=False, threads=0) -> bytes:
    """G1 transform of len(points) / (64 n) rows of n points (arkworks
    Radix2EvaluationDomain fft / ifft over G1, rows normalised to affine)."""
    rows = len(points) // (64 * n)
    out = _buf(64 * n * rows)
    assert lib().oracle_g1_fft(points, n, rows, int(inverse), out, threads) == 0
    return out.raw


def g1_scale(points: bytes, scalars: bytes, threads=0) -> bytes:
    """[s_i] P_i for each point (wire form)."""
    n = len(scalars) // 32
    assert len(points) == 64 * n
    out = _buf(max(1, 64 * n))
    if lib().oracle_g1_scale(points, scalars, n, out, threads) != 0:
        raise ValueError("oracle: bad point or scalar")
    return out.raw[:64 * n]


def ntt(values: bytes, kind="forward") -> bytes:
    buf = ctypes.create_string_buffer(bytes(values), len(values))
    if lib().oracle_ntt(buf, len(values) // 32, NTT_KINDS[kind]) != 0:
        raise ValueError("oracle: bad NTT input")
    return buf.raw


def fixed_base_g1(scalars: bytes, threads=0) -> bytes:
    n = len(scalars) // 32
    out = _buf(64 * n)
    lib().oracle_fixed_base_g1(scalars, n, out, threads)
    return out.raw


def fixed_base_g2(scalars: bytes, threads=0) -> bytes:
    n = len(scalars) // 32
    out = _buf(128 * n)
    lib().oracle_fixed_base_g2(scalars, n, out, threads)
    return out.raw


def g2_check(wire: bytes, algorithm=1, threads=0):
    n = len(wire) // 128
    masks = np.zeros(n, dtype=np.uint32)
    lib().oracle_g2_check(wire, n, algorithm, masks.ctypes.data, threads)
    return masks


def uniform_fr(seed: int, n: int) -> bytes:
    out = _buf(32 * n)
    lib().oracle_chacha_uniform(seed, n, 0, out)
    return out.raw


def uniform_fq(seed: int, n: int) -> bytes:
    out = _buf(32 * n)
    lib().oracle_chacha_uniform(seed, n, 1, out)
    return out.raw


def fr_powers(tau: bytes, n: int) -> bytes:
    out = _buf(32 * n)
    lib().oracle_fr_powers(tau, n, out)
    return out.raw


def g2_twist_points(seed: int, n: int) -> bytes:
    out = _buf(128 * n)
    got = lib().oracle_g2_twist_points(seed, n, out)
    assert got == n
    return out.raw


def g1_add(a: bytes, b: bytes) -> bytes:
    out = _buf(64)
    assert lib().oracle_g1_add(a, b, out) == 0
    return out.raw


def g2_add(a: bytes, b: bytes) -> bytes:
    out = _buf(128)
    assert lib().oracle_g2_add(a, b, out) == 0
    return out.raw


def g2_mul_r(a: bytes) -> bytes:
    out = _buf(128)
    assert lib().oracle_g2_mul_r(a, out) == 0
    return out.raw


def g1_on_curve(p: bytes) -> bool:
    return bool(lib().oracle_g1_on_curve(p))


def g2_on_curve(p: bytes) -> bool:
    return bool(lib().oracle_g2_on_curve(p))


def srs_g1(seed: int, n: int, threads=0):
    """[tau^i]G1 for a seeded uniform tau; returns (points, tau_bytes)."""
    tau = uniform_fr(seed, 1)
    return fixed_base_g1(fr_powers(tau, n), threads), tau


def srs_g2(seed: int, n: int, threads=0):
    tau = uniform_fr(seed, 1)
    return fixed_base_g2(fr_powers(tau, n), threads), tau


# ---------------------------------------------------------------- polynomial toolkit
# Restatement of crates/protocol/src/domain/fast.rs (bn254_oracle.cpp):
# coefficient vectors are canonical Fr bytes, lowest degree first, trimmed.
def poly_mul(left: bytes, right: bytes) -> bytes:
    out = _buf(max(32, len(left) + len(right)))
    n = lib().oracle_poly_mul(left, len(left) // 32, right, len(right) // 32, out)
    return out.raw[:32 * n]


def poly_div_exact(numerator: bytes, denominator: bytes) -> bytes:
    """Quotient of an exact division; ValueError with the reference's message
    otherwise (domain/fast.rs:163-170, 236-240)."""
    out = _buf(max(32, len(numerator)))
    n = ctypes.c_size_t()
    rc = lib().oracle_poly_div_exact(numerator, len(numerator) // 32, denominator, len(denominator) // 32, out,
                                     ctypes.byref(n))
    if rc == -2:
        raise ValueError("cannot divide by zero polynomial")
    if rc == -3:
        raise ValueError("polynomial division has a nonzero remainder")
    if rc != 0:
        raise ValueError("oracle: bad polynomial input")
    return out.raw[:32 * n.value]


class Tree:
    """SubproductTree (domain/fast.rs:11-139) over canonical Fr points."""

    def __init__(self, points: bytes):
        self.n = len(points) // 32
        self._h = lib().oracle_tree_new(points, self.n)
        if not self._h:
            raise ValueError("duplicate interpolation point")

    def close(self):
        if self._h:
            lib().oracle_tree_free(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def vanishing(self) -> bytes:
        out = _buf(32 * (self.n + 1))
        k = lib().oracle_tree_vanishing(self._h, out)
        return out.raw[:32 * k]

    def inverse_derivatives(self) -> bytes:
        out = _buf(max(32, 32 * self.n))
        lib().oracle_tree_inverse_derivatives(self._h, out)
        return out.raw[:32 * self.n]

    def multipoint_eval(self, poly: bytes) -> bytes:
        out = _buf(max(32, 32 * self.n))
        assert lib().oracle_tree_eval(self._h, poly, len(poly) // 32, out) == 0
        return out.raw[:32 * self.n]

    def interpolate(self, values: bytes) -> bytes:
        assert len(values) == 32 * self.n
        out = _buf(max(32, 32 * self.n))
        k = lib().oracle_tree_interpolate(self._h, values, out)
        return out.raw[:32 * k]

    def cauchy_sums(self, weights: bytes) -> bytes:
        assert len(weights) == 32 * self.n
        out = _buf(max(32, 32 * self.n))
        lib().oracle_tree_cauchy(self._h, weights, out)
        return out.raw[:32 * self.n]


# ---------------------------------------------------------------- pairing
# Optimal ate pairing and product checks (crates/protocol/src/verification.rs:37-144).
def pairing(g1: bytes, g2: bytes, threads=0) -> bytes:
    """e(P_i, Q_i) for concatenated G1 (64 B) and G2 (128 B) points: 384-byte
    GT elements in tower order."""
    n = len(g1) // 64
    assert len(g2) == 128 * n
    out = _buf(max(1, 384 * n))
    if lib().oracle_pairing(g1, g2, n, out, threads) != 0:
        raise ValueError("oracle: invalid pairing input")
    return out.raw[:384 * n]


def pairing_check(g1: bytes, g2: bytes, offsets, threads=0):
    """Verdicts of prod_{k in [offsets[e], offsets[e+1])} e(P_k, Q_k) == 1."""
    off = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
    eqs = len(off) - 1
    out = _buf(max(1, eqs))
    if lib().oracle_pairing_check(g1, g2, off.ctypes.data, eqs, out, threads) != 0:
        raise ValueError("oracle: invalid pairing input")
    return [bool(x) for x in out.raw[:eqs]]
