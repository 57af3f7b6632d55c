"""The Dynaverse protocol oracle (oracle/dynaverse.py) on the CPU.

Pins the oracle's two routes to each other and to the properties the
reference's own tests assert, since arkworks cannot run here:
  * srs.rs:219-285: sparse small-domain Lagrange / opening / public-quotient
    bases equal the dense KZG commitments of the interpolated polynomials;
  * dynaverse.rs:1253-1272: cached single openings combine to the dense
    batch opening;
  * dynaverse/sparse_tests.rs:6-41: sparse delta proofs for affected sets of
    size 0, 1, 3, n - 1 and n verify (the bases route follows sparse.rs
    step by step; the scalar route evaluates the dense definitions of
    prove_delta, dynaverse.rs:545-747, at the trapdoor -- their agreement is
    the reference's "sparse == dense" assertion);
  * dynaverse/sparse_tests.rs:57-88: a session through hotspot edits, a
    public-input change, a revert and a synchronous rebuild, every proof
    verified;
  * dynaverse/sparse_tests.rs:90-115: invalid updates are rejected with no
    state change, no-ops return the current proof;
  * the verifier rejects a proof with any single field replaced.
"""
import pytest

from oracle import dynaverse as D
from oracle import oracle as O

R = D.R


@pytest.fixture(scope="module")
def params8():
    tx, ty = D.sample_trapdoors(51, 8)
    return D.Params(8, tx, ty, "bases"), D.Params(8, tx, ty, "scalar")


def _affected_update(n, w, count, seed):
    vals = D.ints(O.uniform_fr(seed, max(1, count)))
    cur = list(w)
    for i in range(count):
        cur[4 * n + i] = (cur[4 * n + i] + vals[i]) % R
        cur[5 * n + i] = cur[3 * n + i] * cur[4 * n + i] % R
    return cur


def test_sparse_bases_equal_dense_commitments(params8):
    pb, _ = params8
    n, m = pb.n, pb.m
    vals = D.ints(O.uniform_fr(61, n))
    coeffs = D.ints(O.ntt(D.frs(vals), "inverse"))
    assert pb.gather("lag", list(enumerate(vals))) == pb.commit(coeffs)
    assert O.msm_g2(b"".join(pb.lag_g2), D.frs(vals)) == pb.commit_g2(coeffs)
    for i in (0, n // 2, n - 1):
        unit = [0] * n
        unit[i] = 1
        num = D.ints(O.ntt(D.frs(unit), "inverse"))
        num[0] = (num[0] - 1) % R
        q = D.ints(O.poly_div_exact(D.frs(num), D.frs([(-pb.small_points[i]) % R, 1])))
        assert pb.B["open_u"][i] == pb.commit(q)
    big = [0] * m
    for i in (0, n - 1, 3 * n, 6 * n - 1):
        big[i] = D.ints(O.uniform_fr(62 + i, 1))[0]
    coeffs = D.ints(O.ntt(D.frs(big), "inverse"))
    ix = [1]
    for i in range(6 * n, m):
        ix = D._pmul(ix, [(-pow(pb.wm, i, R)) % R, 1])
    q = D.ints(O.poly_div_exact(D.frs(coeffs), D.frs(ix)))
    assert pb.gather("pq", [(i, v) for i, v in enumerate(big) if v]) == pb.commit(q)


def test_routes_agree_on_anchor_cache_and_verify(params8):
    pb, ps = params8
    pub, w = D.valid_instance(pb.n)
    a_b, a_s = pb.prove_anchor(w), ps.prove_anchor(w)
    assert a_b.to_bytes() == a_s.to_bytes()
    assert pb.opening_cache(w) == ps.opening_cache(w)
    proof = D.Proof(a_b, None, 0, 0)
    assert pb.verify(pub, proof) and ps.verify(pub, proof)


def test_cached_openings_combine_to_dense_batch_opening(params8):
    pb, _ = params8
    n = pb.n
    pub, w = D.valid_instance(n)
    cache = pb.opening_cache(w)
    for t in range(3):
        vals = w[(t + 3) * n:(t + 4) * n]
        coeffs = D.ints(O.ntt(D.frs(vals), "inverse"))
        for aff in ([0], [1, 7], [2, 3, 5]):
            pts = [pb.small_points[i] for i in aff]
            with O.Tree(D.frs(pts)) as tree:
                weights = D.ints(tree.inverse_derivatives())
                r = D.ints(tree.interpolate(D.frs([vals[i] for i in aff])))
                a = D.ints(tree.vanishing())
            combined = O.msm_g1(b"".join(cache[t][i] for i in aff), D.frs(weights))
            q = D.ints(O.poly_div_exact(D.frs(D._psub(coeffs, r)), D.frs(a)))
            assert combined == pb.commit(q)


@pytest.mark.parametrize("n", [2, 8, 16])
def test_sparse_delta_routes_agree_and_verify_for_every_affected_size(n):
    tx, ty = D.sample_trapdoors(100 + n, n)
    pb, ps = D.Params(n, tx, ty, "bases"), D.Params(n, tx, ty, "scalar")
    pub, anchor = D.valid_instance(n)
    a = pb.prove_anchor(anchor)
    cache = pb.opening_cache(anchor)
    for count in sorted({0, 1, min(3, n), n - 1, n}):
        cur = _affected_update(n, anchor, count, 200 + n + count)
        new_pub = list(pub)
        if count == 0:  # an edit outside the multiplication wires (sparse_tests.rs:20-23)
            cur[1] = (cur[1] + 1) % R
            cur[n + 1] = (cur[n + 1] - 1) % R
        new_pub[1] = cur[1]
        entries = [(i, (x - y) % R) for i, (x, y) in enumerate(zip(cur, anchor)) if x != y]
        d_b = pb.prove_delta(anchor, entries, a.wires, cache)
        d_s = ps.prove_delta(anchor, entries, a.wires, None)
        assert d_b.to_bytes() == d_s.to_bytes(), f"n={n} a={count}"
        proof = D.Proof(a, d_b, 0, 1)
        assert pb.verify(new_pub, proof), f"n={n} a={count}"
        assert D.parse_proof(proof.to_bytes()).to_bytes() == proof.to_bytes()


def test_verifier_rejects_any_replaced_field(params8):
    pb, _ = params8
    n = pb.n
    pub, anchor = D.valid_instance(n)
    a = pb.prove_anchor(anchor)
    cache = pb.opening_cache(anchor)
    cur = _affected_update(n, anchor, 3, 77)
    entries = [(i, (x - y) % R) for i, (x, y) in enumerate(zip(cur, anchor)) if x != y]
    good = D.Proof(a, pb.prove_delta(anchor, entries, a.wires, cache), 0, 1).to_bytes()
    assert pb.verify(pub, D.parse_proof(good))
    g = D.g1_gen()
    # replace G1 fields across the anchor and the delta (offsets of 64-byte slots)
    for off in (0, 6 * 64 + 128, 3968, 3968 + 9 * 64, 3968 + 59 * 64, D.PROOF_BYTES - 24 - 64):
        bad = bytearray(good)
        bad[off:off + 64] = g if bytes(bad[off:off + 64]) != g else bytes(64)
        assert not pb.verify(pub, D.parse_proof(bytes(bad))), off
    bad = bytearray(good)
    bad[3968 + 60 * 64] ^= 1  # affected_g2 moved off the twist curve
    assert not pb.verify(pub, D.parse_proof(bytes(bad)))
    wrong_pub = list(pub)
    wrong_pub[0] = (wrong_pub[0] + 1) % R
    assert not pb.verify(wrong_pub, D.parse_proof(good))


def _session_steps(n, w):
    """The edit sequence of session_matches_dense_through_hotspots_reverts_
    public_changes_and_rebuilds (sparse_tests.rs:57-88)."""
    steps = []
    for step in range(12):
        if step == 4:
            steps.append(("public", 1))
        else:
            i = 1 if step < 4 else step - 4
            steps.append(("mul", i, step == 3))
    return steps


def test_session_routes_agree_through_hotspots_public_revert_and_rebuild():
    n = 16
    tx, ty = D.sample_trapdoors(15301, n)
    pb, ps = D.Params(n, tx, ty, "bases"), D.Params(n, tx, ty, "scalar")
    pub, w = D.valid_instance(n)
    sb, ss = D.Session(pb, pub, w), D.Session(ps, pub, w)
    assert sb.proof.to_bytes() == ss.proof.to_bytes()
    original = list(w)
    rebuilt = False
    for kind, i, *rest in _session_steps(n, w):
        cur = sb.current
        if kind == "public":
            new = (sb.pub[i] + 1) % R
            args = ([i, n + i], [(cur[i] + 1) % R, (cur[n + i] - 1) % R], [i], [new])
        else:
            value = original[4 * n + i] if rest[0] else (cur[4 * n + i] + 1) % R
            args = ([4 * n + i, 5 * n + i], [value, cur[3 * n + i] * value % R], [], [])
        pb_proof = sb.update(*args)
        ps_proof = ss.update(*args)
        assert pb_proof.to_bytes() == ps_proof.to_bytes()
        assert sb.current == ss.current and sb.pub == ss.pub
        rebuilt |= pb_proof.delta is None
    assert rebuilt and sb.proof.anchor_generation > 0


def test_session_rejects_invalid_updates_and_keeps_noops():
    n = 8
    tx, ty = D.sample_trapdoors(15302, n)
    ps = D.Params(n, tx, ty, "scalar")
    pub, w = D.valid_instance(n)
    s = D.Session(ps, pub, w)
    before = s.proof.to_bytes()
    for idx, vals in (([6 * n], [1]), ([0], []), ([n + 1], [0]), ([3 * n + 1], [0]), ([5 * n + 1], [0])):
        with pytest.raises(ValueError):
            s.update(idx, vals)
        assert s.proof.to_bytes() == before and s.current == w and s.pub == pub and s.anchor_distance() == 0
    assert s.update([4 * n + 1, 4 * n + 1], [0, w[4 * n + 1]]).to_bytes() == before
    with pytest.raises(ValueError):
        s.update([], [], [1], [0])
    assert s.pub == pub
