"""Resident transactional buffers (dvgpu_resident_*) against a model of the
reference's CPU RebuildBackend (crates/protocol/src/incremental_rebuild/
operators.rs:113-500): the same randomised sequence of writes, copies,
transposes, row transforms, zips, scalings, MSMs, commits and rollbacks runs
on the GPU engine and on the model (field arithmetic in Python integers,
group arithmetic and transforms from the oracle), and every buffer is
compared after every transaction."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
ROOT28 = 0x2A3C09F0A58A7E8500E0A7EB8EF62ABC402D111E41112ED49BD61B6E725B19F0
FR, G1, BASES = 0, 1, 2
INF = bytes(64)


def fr_bytes(v):
    return (v % R).to_bytes(32, "little")


class Model:
    """operators.rs CpuRebuildBackend: buffers, first-write undo journal."""

    def __init__(self, oracle):
        self.o = oracle
        self.bufs = []  # [kind, values, writable, saved]
        self.sealed = False
        self.tx = False
        self.undo = []

    def alloc(self, kind, n, writable):
        assert not self.sealed and not self.tx
        self.bufs.append([kind, [0 if kind == FR else INF] * n, writable, [False] * n])
        return len(self.bufs) - 1

    def _check(self, h, kind, off, n, write):
        k, vals, writable, _ = self.bufs[h]
        if k != kind or off + n > len(vals) or (write and self.sealed and not writable):
            raise ValueError("invalid")

    def _put(self, h, i, v):
        b = self.bufs[h]
        if self.tx and not b[3][i]:
            self.undo.append((h, i, b[1][i]))
            b[3][i] = True
        b[1][i] = v

    @staticmethod
    def _alias(src, so, dst, do, n, exact):
        if src != dst or n == 0:
            return
        if so < do + n and do < so + n and not (exact and so == do):
            raise ValueError("alias")

    def begin(self):
        if self.tx:
            raise ValueError("active")
        self.tx = True

    def commit(self):
        for h, i, _ in self.undo:
            self.bufs[h][3][i] = False
        self.undo, self.tx = [], False

    def rollback(self):
        if not self.tx:
            raise ValueError("none")
        while self.undo:
            h, i, old = self.undo.pop()
            self.bufs[h][1][i] = old
            self.bufs[h][3][i] = False
        self.tx = False

    def write(self, h, off, vals, kind):
        self._check(h, kind, off, len(vals), True)
        for j, v in enumerate(vals):
            self._put(h, off + j, v)

    def copy(self, src, so, dst, do, n, reverse=False, kind=None):
        kind = self.bufs[src][0] if kind is None else kind
        self._check(src, kind, so, n, False)
        self._check(dst, kind, do, n, True)
        self._alias(src, so, dst, do, n, n <= 1 if reverse else True)
        vals = list(self.bufs[src][1][so:so + n])
        if reverse:
            vals = vals[::-1]
        for j, v in enumerate(vals):
            self._put(dst, do + j, v)

    def _smul(self, p, k):
        return self.o.msm_g1(p, fr_bytes(k))

    def transpose(self, kind, src, dst, rows, cols, start, n, root):
        size = rows * cols
        if start + n > size:
            raise ValueError("range")
        self._check(src, kind, 0, size, False)
        self._check(dst, kind, 0, size, True)
        if src == dst and n:
            raise ValueError("distinct")
        for i in range(start, start + n):
            row, col = divmod(i, cols)
            v = self.bufs[src][1][i]
            if root is not None:
                f = pow(root, row * col, R)
                v = v * f % R if kind == FR else self._smul(v, f)
            self._put(dst, col * rows + row, v)

    def transform_rows(self, kind, src, dst, row_len, first, count, inverse):
        start, n = first * row_len, count * row_len
        self._check(src, kind, start, n, False)
        self._check(dst, kind, start, n, True)
        if src == dst and n:
            raise ValueError("distinct")
        for r in range(count):
            row = self.bufs[src][1][start + r * row_len:start + (r + 1) * row_len]
            if kind == FR:
                out = self.o.ntt(b"".join(fr_bytes(v) for v in row), "inverse" if inverse else "forward")
                res = [int.from_bytes(out[32 * j:32 * (j + 1)], "little") for j in range(row_len)]
            else:
                out = self.o.g1_fft(b"".join(row), row_len, inverse)
                res = [out[64 * j:64 * (j + 1)] for j in range(row_len)]
            for j, v in enumerate(res):
                self._put(dst, start + r * row_len + j, v)

    def zip(self, op, a, ao, b, bo, c, co, n):
        self._check(a, FR, ao, n, False)
        self._check(b, FR, bo, n, False)
        self._check(c, FR, co, n, True)
        self._alias(a, ao, c, co, n, True)
        self._alias(b, bo, c, co, n, True)
        for j in range(n):
            x, y = self.bufs[a][1][ao + j], self.bufs[b][1][bo + j]
            self._put(c, co + j, (x + y, x - y, x * y)[op] % R)

    def scale(self, p, po, s, so, d, do, n):
        self._check(p, G1, po, n, False)
        self._check(s, FR, so, n, False)
        self._check(d, G1, do, n, True)
        self._alias(p, po, d, do, n, True)
        res = [self._smul(self.bufs[p][1][po + j], self.bufs[s][1][so + j]) for j in range(n)]
        for j, v in enumerate(res):
            self._put(d, do + j, v)

    def msm_g1(self, p, po, s, so, n):
        pts = b"".join(self.bufs[p][1][po:po + n])
        return self.o.msm_g1(pts, b"".join(fr_bytes(v) for v in self.bufs[s][1][so:so + n]))


def _root20():
    return fr_bytes(pow(ROOT28, 2 ** 8, R))


def _read_all(b, model, handles):
    for mh, (gh, kind) in handles.items():
        vals = model.bufs[mh][1]
        got = b.rb_read(gh, 0, len(vals), FR if kind == FR else G1)
        exp = b"".join(fr_bytes(v) for v in vals) if kind == FR else b"".join(vals)
        assert got == exp, f"buffer {mh} (kind {kind})"


def test_resident_transactions_match_cpu_model(oracle, dv):
    rng = np.random.default_rng(2027)
    b = dv.DvgpuBackend()
    m = Model(oracle)
    try:
        b.resident_configure(1 << 30, 4096 * 144, _root20())
        handles = {}

        def alloc(kind, n, writable):
            g, h = b.rb_alloc(kind, n, writable), m.alloc(kind, n, writable)
            handles[h] = (g, kind)
            assert b.rb_len(g) == n and b.rb_kind(g) == kind
            return h

        F = [alloc(FR, 64, True) for _ in range(3)]
        F_ro = alloc(FR, 64, False)
        P = [alloc(G1, 16, True) for _ in range(3)]
        P_ro = alloc(G1, 16, False)
        pts, _ = oracle.srs_g1(3300, 16)
        bases_g = b.rb_register_bases(pts)
        assert b.rb_kind(bases_g) == BASES
        G = lambda h: handles[h][0]

        def rand_fr(n, seed):
            raw = oracle.uniform_fr(seed, n)
            return [int.from_bytes(raw[32 * j:32 * (j + 1)], "little") for j in range(n)]

        def rand_pts(n, seed):
            raw, _ = oracle.srs_g1(seed, n)
            return [raw[64 * j:64 * (j + 1)] for j in range(n)]

        for j, h in enumerate(F + [F_ro]):
            v = rand_fr(64, 3400 + j)
            m.write(h, 0, v, FR)
            b.rb_write(G(h), 0, b"".join(fr_bytes(x) for x in v), FR)
        for j, h in enumerate(P + [P_ro]):
            v = rand_pts(16, 3500 + j)
            v[3] = INF
            m.write(h, 0, v, G1)
            b.rb_write(G(h), 0, b"".join(v), G1)
        m.sealed = True
        b.rb_seal()
        _read_all(b, m, handles)

        def both(fn_model, fn_gpu, expect_error=False):
            err_m = err_g = None
            try:
                fn_model()
            except ValueError as e:
                err_m = e
            try:
                fn_gpu()
            except dv.DvgpuError as e:
                err_g = e
                assert e.status == -1, e
            assert (err_m is None) == (err_g is None), (err_m, err_g)
            assert (err_m is not None) == expect_error

        seed = 3600
        for t in range(10):
            m.begin()
            b.rb_begin()
            for _ in range(int(rng.integers(2, 6))):
                seed += 1
                kind_op = int(rng.integers(0, 9))
                f0, f1 = [F[int(i)] for i in rng.choice(3, 2, replace=False)]
                p0, p1 = P[0], P[1]
                if kind_op == 0:
                    off, n = int(rng.integers(0, 60)), int(rng.integers(1, 5))
                    v = rand_fr(n, seed)
                    both(lambda: m.write(f0, off, v, FR), lambda: b.rb_write(G(f0), off, b"".join(map(fr_bytes, v)), FR))
                elif kind_op == 1:
                    off, n = int(rng.integers(0, 12)), int(rng.integers(1, 4))
                    v = rand_pts(n, seed)
                    both(lambda: m.write(p0, off, v, G1), lambda: b.rb_write(G(p0), off, b"".join(v), G1))
                elif kind_op == 2:
                    so, do, n = int(rng.integers(0, 32)), int(rng.integers(0, 32)), int(rng.integers(1, 32))
                    src, dst = (f0, f1) if rng.integers(2) else (f0, f0)
                    rev = bool(rng.integers(2))
                    overlap = src == dst and so < do + n and do < so + n and not (not rev and so == do) \
                        and not (rev and n <= 1)
                    both(lambda: m.copy(src, so, dst, do, n, rev, FR),
                         (lambda: b.rb_reverse(FR, G(src), so, G(dst), do, n)) if rev else
                         (lambda: b.rb_copy(G(src), so, G(dst), do, n)), overlap)
                elif kind_op == 3:
                    start, n = int(rng.integers(0, 32)), int(rng.integers(1, 32))
                    root = int.from_bytes(oracle.uniform_fr(seed, 1), "little") if rng.integers(2) else None
                    both(lambda: m.transpose(FR, f0, f1, 8, 8, start, n, root),
                         lambda: b.rb_transpose(FR, G(f0), G(f1), 8, 8, start, n, None if root is None else fr_bytes(root)))
                elif kind_op == 4:
                    start, n = int(rng.integers(0, 8)), int(rng.integers(1, 9))
                    root = int.from_bytes(oracle.uniform_fr(seed, 1), "little") if rng.integers(2) else None
                    both(lambda: m.transpose(G1, p0, p1, 4, 4, start, n, root),
                         lambda: b.rb_transpose(G1, G(p0), G(p1), 4, 4, start, n, None if root is None else fr_bytes(root)))
                elif kind_op == 5:
                    first, count, inv = int(rng.integers(0, 4)), int(rng.integers(1, 5)), bool(rng.integers(2))
                    over = (first + count) * 8 > 64
                    both(lambda: m.transform_rows(FR, f0, f1, 8, first, count, inv),
                         lambda: b.rb_transform_rows(FR, G(f0), G(f1), 8, first, count, inv), over)
                elif kind_op == 6:
                    first, count, inv = int(rng.integers(0, 2)), int(rng.integers(1, 3)), bool(rng.integers(2))
                    both(lambda: m.transform_rows(G1, p0, p1, 4, first, count, inv),
                         lambda: b.rb_transform_rows(G1, G(p0), G(p1), 4, first, count, inv))
                elif kind_op == 7:
                    op, n = int(rng.integers(0, 3)), int(rng.integers(1, 20))
                    ao, bo = int(rng.integers(0, 40)), int(rng.integers(0, 40))
                    both(lambda: m.zip(op, f0, ao, f1, bo, f0, ao, n),
                         lambda: b.rb_zip(op, G(f0), ao, G(f1), bo, G(f0), ao, n))
                else:
                    po, so, n = int(rng.integers(0, 8)), int(rng.integers(0, 50)), int(rng.integers(1, 8))
                    both(lambda: m.scale(p0, po, f0, so, p1, po, n),
                         lambda: b.rb_scale(G(p0), po, G(f0), so, G(p1), po, n))
            if rng.integers(3) == 0:
                m.rollback()
                b.rb_rollback()
            else:
                m.commit()
                b.rb_commit()
            _read_all(b, m, handles)
            # MSMs read resident buffers, G1 and registered bases
            assert b.rb_msm_g1(G(P[0]), 0, G(F[0]), 10, 16) == m.msm_g1(P[0], 0, F[0], 10, 16)
            assert b.rb_msm_g1(bases_g, 2, G(F[1]), 0, 14) == oracle.msm_g1(
                pts[128:], b"".join(fr_bytes(v) for v in m.bufs[F[1]][1][:14]))

        # packets: a complete transform of one buffer range into another
        b.rb_begin()
        m.begin()
        for kind, src, scr, dst, n, inv in ((FR, F[0], F[2], F[1], 64, False), (G1, P[0], P[2], P[1], 16, True)):
            m.transform_rows(kind, src, dst, n, 0, 1, inv)
            b.rb_transform_packet(kind, G(src), G(scr), G(dst), n, inv)
        m.commit()
        b.rb_commit()
        _read_all(b, m, handles)
        # G2 MSM over host bases with resident scalars
        g2, _ = oracle.srs_g2(3700, 8)
        assert b.rb_msm_g2(g2, G(F[2]), 5) == oracle.msm_g2(g2, b"".join(fr_bytes(v) for v in m.bufs[F[2]][1][5:13]))

        # rule checks: read-only after seal, packed handles, transactions
        with pytest.raises(dv.DvgpuError):
            b.rb_write(G(F_ro), 0, fr_bytes(1), FR)
        with pytest.raises(dv.DvgpuError):
            b.rb_copy(bases_g, 0, G(P[0]), 0, 1)
        with pytest.raises(dv.DvgpuError):
            b.rb_rollback()
        with pytest.raises(dv.DvgpuError):
            b.rb_alloc(FR, 4, True)  # after seal
        b.rb_begin()
        with pytest.raises(dv.DvgpuError):
            b.rb_begin()
        b.rb_zip(2, G(F[0]), 0, G(F[1]), 0, G(F[0]), 0, 64)
        b.rb_rollback()
        _read_all(b, m, handles)  # the rolled-back zip left no trace
        st = b.rb_stats()
        assert st.calls > 0 and st.fr_transform_elements > 0 and st.msm_g1_points > 0
    finally:
        b.close()
    other = dv.DvgpuBackend()
    try:
        with pytest.raises(dv.DvgpuError):
            other.resident_configure(1 << 30, 1 << 20, fr_bytes(5))  # not a root of order 2^20
        other.resident_configure(1 << 30, 64 * 144, _root20())  # a journal of 64 records
        f = other.rb_alloc(FR, 128, True)
        other.rb_seal()
        other.rb_begin()
        other.rb_write(f, 0, bytes(32 * 64), FR)
        other.rb_write(f, 0, fr_bytes(7), FR)  # already saved: no new record
        with pytest.raises(dv.DvgpuError) as e:  # the 65th first write
            other.rb_write(f, 64, fr_bytes(1), FR)
        assert e.value.status == -1 and "journal" in e.value.message
        other.rb_rollback()
        assert other.rb_read(f, 0, 128, FR) == bytes(32 * 128)
    finally:
        other.close()
