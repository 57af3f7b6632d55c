"""Serving engine parity on the GPU (dvgpu_serve_*).

Every served commitment must equal the oracle's full recommitment of the
updated vector (sum v_i G_i over the session's SRS), and every request must
get the same result in the merged mix as alone (max_batch = 1), the
property the reference's per-session update loop guarantees by running one
update at a time (crates/protocol/src/session.rs:51-142).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


def _sessions(oracle, sizes, seed):
    out = []
    for j, n in enumerate(sizes):
        pts, _ = oracle.srs_g1(seed + j, n)
        out.append((pts, bytearray(oracle.uniform_fr(seed + 100 + j, n))))
    return out


def _requests(oracle, sizes, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for t in range(count):
        s = int(rng.integers(len(sizes)))
        n = sizes[s]
        k = int(min(n, max(1, int(2 ** rng.uniform(0, 7)))))
        if t % 2:  # hotspot: a 64-entry window
            base = int(rng.integers(max(1, n - 64)))
            idx = base + rng.choice(min(64, n), size=min(k, 64, n), replace=False)
        else:
            idx = rng.choice(n, size=k, replace=False)
        vals = oracle.uniform_fr(seed * 1000 + t, len(idx))
        reqs.append((s, [int(i) for i in idx], vals))
    return reqs


def _expected(oracle, sess, reqs):
    vecs = [bytearray(v) for _, v in sess]
    exp = []
    for s, idx, vals in reqs:
        for j, i in enumerate(idx):
            vecs[s][32 * i:32 * (i + 1)] = vals[32 * j:32 * (j + 1)]
        exp.append(oracle.msm_g1(sess[s][0], bytes(vecs[s])))
    return exp


def _serve(dv, sess, reqs, max_batch):
    with dv.DvgpuServer(1 << 30, max_batch) as srv:
        ids, initial = [], []
        for pts, vals in sess:
            sid, c0 = srv.open_session(pts, bytes(vals))
            ids.append(sid)
            initial.append(c0)
        tickets = [srv.submit(ids[s], idx, vals) for s, idx, vals in reqs]
        outs = [srv.wait(t) for t in tickets]
        st = srv.stats()
        return initial, [o[0] for o in outs], [o[1] for o in outs], st


def test_served_commitments_match_oracle_and_per_call(oracle, dv):
    sizes = [256, 300, 1024, 64]
    sess = _sessions(oracle, sizes, 610)
    reqs = _requests(oracle, sizes, 48, 611)
    exp = _expected(oracle, sess, reqs)
    init, merged, res, st = _serve(dv, sess, reqs, 64)
    for j, (pts, vals) in enumerate(sess):
        assert init[j] == oracle.msm_g1(pts, bytes(vals))
    for t in range(len(reqs)):
        assert merged[t] == exp[t], f"request {t}"
    assert st.requests == len(reqs) and st.largest_batch > 1 and st.batches < len(reqs)
    assert all(r.done_ns >= r.start_ns >= r.submit_ns for r in res)
    _, alone, res1, st1 = _serve(dv, sess, reqs, 1)
    assert alone == merged
    assert st1.batches == len(reqs) and all(r.batch_requests == 1 for r in res1)


def test_serve_admission_and_invalid_updates(oracle, dv):
    pts, _ = oracle.srs_g1(620, 512)
    vals = oracle.uniform_fr(621, 512)
    with dv.DvgpuServer(512 * (64 * 33 + 32) + 64, 8) as srv:  # room for exactly one session of 512
        sid, c0 = srv.open_session(pts, vals)
        with pytest.raises(dv.DvgpuError) as e:
            srv.open_session(pts, vals)
        assert e.value.status == -1 and "budget" in e.value.message
        one = oracle.uniform_fr(622, 1)
        bad = (R_MOD).to_bytes(32, "little")
        for idx, v in (([512], one), ([3, 3], one + one), ([4], bad), ([], b"")):
            with pytest.raises(dv.DvgpuError) as e:
                srv.submit(sid, idx, v)
            assert e.value.status == -1
        with pytest.raises(dv.DvgpuError):
            srv.submit(sid + 7, [1], one)
        # the server stays usable; an update that restores the old value gives back C0
        c1, _ = srv.wait(srv.submit(sid, [5], one))
        assert c1 != c0
        c2, _ = srv.wait(srv.submit(sid, [5], vals[32 * 5:32 * 6]))
        assert c2 == c0
        srv.close_session(sid)
        sid2, c0b = srv.open_session(pts, vals)  # the budget is free again
        assert c0b == c0
