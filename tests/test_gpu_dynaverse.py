"""Dynaverse update proofs on the device against the protocol oracle.

Every proof the engine returns is compared byte for byte with the oracle's
proof for the same trapdoors, witness and updates (oracle/dynaverse.py,
scalar route, itself pinned to the reference's steps in
tests/test_oracle_dynaverse.py), and checked by the device verifier.
Mirrors crates/protocol/src/dynaverse/sparse_tests.rs:
  * a session through hotspot edits, a public-input change, a revert and a
    synchronous rebuild (session_matches_dense_through_hotspots_...);
  * affected sets of every size the sparse path admits, the empty one
    included (sparse_delta_matches_every_dense_field_...);
  * invalid updates rejected with no state change, no-ops returning the
    current proof (session_rejects_invalid_updates_atomically_...);
and the workload shapes: the CPU-runnable sequence of n = 256 with 8 hotspot
updates, and a session of n = 65536 through sparse updates and a re-anchor.
Served and per-call forms give identical proofs, and every proof alone
equals the same proof in a mixed batch."""
import numpy as np
import pytest

from oracle import dynaverse as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu
R = D.R
GB = 1 << 30


@pytest.fixture(scope="module")
def engine(dv):
    e = dv.DynaverseEngine(120 * GB, 64)
    yield e
    e.close()


def _setup(engine, n, seed):
    tx, ty = D.sample_trapdoors(seed, n)
    return engine.params_create(n, tx, ty), D.Params(n, tx, ty, "scalar")


def _mul_edit(n, cur, gate, value):
    """A circuit-valid edit of the multiplication gate: s5 = value, s6 = s4 * value."""
    return [4 * n + gate, 5 * n + gate], [value % R, cur[3 * n + gate] * value % R]


def test_session_matches_oracle_through_hotspots_public_revert_and_rebuild(engine, dv):
    n = 16
    ph, P = _setup(engine, n, 15301)
    pub, w = D.valid_instance(n)
    s, proof = engine.open_session(ph, pub, w)
    ref = D.Session(P, pub, w)
    assert proof == ref.proof.to_bytes()
    assert engine.verify(ph, pub, proof)
    original = list(w)
    kinds = set()
    for step in range(12):
        cur = ref.current
        if step == 4:
            new = (ref.pub[1] + 1) % R
            args = ([1, n + 1], [(cur[1] + 1) % R, (cur[n + 1] - 1) % R], [1], [new])
        else:
            i = 1 if step < 4 else step - 4
            value = original[4 * n + i] if step == 3 else cur[4 * n + i] + 1
            args = (*_mul_edit(n, cur, i, value), [], [])
        expect = ref.update(*args).to_bytes()
        got = engine.update(s, *args)
        assert got == expect, f"step {step}"
        assert engine.verify(ph, ref.pub, got)
        kinds.add(D.parse_proof(got).delta is None)
        wit, pb, cur_proof, dist = engine.session_state(s, n)
        assert D.ints(wit) == ref.current and D.ints(pb) == ref.pub and cur_proof == expect
        assert dist == ref.anchor_distance()
    assert kinds == {True, False}  # both sparse proofs and a re-anchor
    engine.close_session(s)


def test_every_affected_size_and_the_empty_set(engine):
    n = 64  # rebuild interval 8: deltas of up to 7 entries stay sparse
    ph, P = _setup(engine, n, 15401)
    pub, w = D.valid_instance(n)
    vals = D.ints(O.uniform_fr(15402, 16))
    for count in (0, 1, 2, 3):
        s, _ = engine.open_session(ph, pub, w)
        ref = D.Session(P, pub, w)
        if count == 0:  # a public-input change that leaves the multiplication wires alone
            args = ([1, n + 1], [(w[1] + 1) % R, (w[n + 1] - 1) % R], [1], [(pub[1] + 1) % R])
        else:
            idx, v = [], []
            for g in range(count):
                ii, vv = _mul_edit(n, w, 3 * g + 2, vals[g])
                idx += ii
                v += vv
            args = (idx, v, [], [])
        expect = ref.update(*args)
        assert expect.delta is not None
        got = engine.update(s, *args)
        assert got == expect.to_bytes(), count
        assert engine.verify(ph, ref.pub, got)
        engine.close_session(s)


def test_invalid_updates_are_rejected_without_state_change(engine, dv):
    n = 32
    ph, _ = _setup(engine, n, 15302)
    pub, w = D.valid_instance(n)
    s, before = engine.open_session(ph, pub, w)
    cases = [([6 * n], [1], "out of range"), ([n + 1], [0], "addition gate fails at 1"),
             ([3 * n + 1], [0], "wire copy constraint fails at 1"),
             ([5 * n + 1], [0], "multiplication gate fails at 1")]
    for idx, vals, msg in cases:
        with pytest.raises(dv.DvgpuError) as e:
            engine.update(s, idx, vals)
        assert e.value.status == -1 and msg in e.value.message
        wit, pb, proof, dist = engine.session_state(s, n)
        assert proof == before and D.ints(wit) == w and D.ints(pb) == pub and dist == 0
    with pytest.raises(dv.DvgpuError):
        engine.update(s, [], [], [1], [0])  # public copy constraint
    assert engine.update(s, [4 * n + 1, 4 * n + 1], [0, w[4 * n + 1]]) == before  # no-op
    # the verifier rejects a changed field and a wrong instance
    assert engine.verify(ph, pub, before)
    bad = bytearray(before)
    bad[64 * 3:64 * 4] = bad[0:64]
    assert not engine.verify(ph, pub, bytes(bad))
    wrong = list(pub)
    wrong[0] = (wrong[0] + 1) % R
    assert not engine.verify(ph, wrong, before)
    engine.close_session(s)


def test_served_batches_equal_per_call_proofs(engine, dv):
    """Sessions of two sizes, several updates each, submitted at once: the
    merged batches return the proofs the oracle computes one update at a
    time (the same in the mix as alone)."""
    specs = [(16, 700), (16, 701), (64, 702), (64, 703), (256, 704)]
    rng = np.random.default_rng(705)
    sessions = []
    for n, seed in specs:
        ph, P = _setup(engine, n, seed)
        pub, w = D.valid_instance(n)
        s, _ = engine.open_session(ph, pub, w)
        sessions.append((n, s, D.Session(P, pub, w)))
    expected, updates = {}, []
    for step in range(3):
        for k, (n, s, ref) in enumerate(sessions):
            gates = rng.choice(n, size=1 + step % 2, replace=False)
            vals = D.ints(O.uniform_fr(800 + 10 * k + step, len(gates)))
            idx, v = [], []
            for g, val in zip(gates, vals):
                ii, vv = _mul_edit(n, ref.current, int(g), val)
                idx += ii
                v += vv
            expected[(k, step)] = ref.update(idx, v).to_bytes()
            updates.append(((k, step), s, idx, v))
    # all submitted at once: while one batch is on the GPU the rest queue up
    tickets = [(key, engine.submit(s, idx, v)) for key, s, idx, v in updates]
    batches = set()
    for key, t in tickets:
        proof, res = engine.wait(t)
        assert proof == expected[key], key
        batches.add(res.batch_id)
    assert len(batches) < len(tickets)  # updates of different sessions shared batches
    for n, s, _ in sessions:
        engine.close_session(s)


def test_cpu_sequence_shape_n256_eight_hotspot_updates(engine):
    """The CPU-runnable sequence: n = 256, 8 updates, each rewriting 4
    indices of a 16-gate hotspot with fresh uniform values (2 gates, wires
    s5 and s6, so the circuit stays valid), re-anchoring when the delta
    reaches ceil(sqrt(256)) = 16."""
    n = 256
    ph, P = _setup(engine, n, 2812)
    pub, w = D.valid_instance(n)
    s, proof = engine.open_session(ph, pub, w)
    ref = D.Session(P, pub, w)
    assert proof == ref.proof.to_bytes()
    rng = np.random.default_rng(2813)
    hot = list(range(40, 56))
    rebuilt = 0
    for step in range(8):
        gates = rng.choice(hot, size=2, replace=False)
        vals = D.ints(O.uniform_fr(2900 + step, 2))
        idx, v = [], []
        for g, val in zip(gates, vals):
            ii, vv = _mul_edit(n, ref.current, int(g), val)
            idx += ii
            v += vv
        expect = ref.update(idx, v)
        assert engine.update(s, idx, v) == expect.to_bytes(), step
        rebuilt += expect.delta is None
    assert rebuilt >= 1
    engine.close_session(s)


def test_n65536_sparse_updates_and_reanchor_match_oracle(engine):
    n = 1 << 16
    ph, P = _setup(engine, n, 65536)
    pub, w = D.valid_instance(n)
    s, proof = engine.open_session(ph, pub, w)
    ref = D.Session(P, pub, w, verify=False)
    assert proof == ref.proof.to_bytes()
    rng = np.random.default_rng(65537)
    # sparse updates: a hotspot window of 64 gates, then uniform gates, until
    # the delta reaches ceil(sqrt(n)) = 256 and the session re-anchors
    hot, every = np.arange(1000, 1064), np.arange(n)
    for step, (pool, k) in enumerate([(hot, 1), (every, 7), (hot, 40), (every, 60), (every, 128)]):
        gates = rng.choice(pool, size=k, replace=False)
        vals = D.ints(O.uniform_fr(66000 + step, len(gates)))
        idx, v = [], []
        for g, val in zip(gates, vals):
            ii, vv = _mul_edit(n, ref.current, int(g), val)
            idx += ii
            v += vv
        expect = ref.update(idx, v, verify=False)
        got = engine.update(s, idx, v)
        assert got == expect.to_bytes(), step
    assert ref.proof.anchor_generation > 0  # the last update re-anchored
    engine.close_session(s)
    engine.params_destroy(ph)


def test_admission_budget_and_lifecycle_rules(dv):
    """HBM admission by measured footprint (parameters and sessions), unknown
    handles, closing a session while its update is queued, and releasing
    parameters that still have sessions: each refused with status -1 and the
    engine still serving afterwards."""
    import threading
    n = 16
    tx, ty = D.sample_trapdoors(15303, n)
    pub, w = D.valid_instance(n)
    with dv.DynaverseEngine(1 << 20, 8) as small:  # below one parameter set of n = 16
        with pytest.raises(dv.DvgpuError) as e:
            small.params_create(n, tx, ty)
        assert e.value.status == -1 and "HBM budget" in e.value.message
    with dv.DynaverseEngine(1 << 30, 8) as probe:
        ph = probe.params_create(n, tx, ty)
        params_bytes = probe.stats().resident_bytes
        s, _ = probe.open_session(ph, pub, w)
        session_bytes = probe.stats().resident_bytes - params_bytes
        probe.close_session(s)
    # room for the parameters and one session: the second session is refused
    with dv.DynaverseEngine(params_bytes + session_bytes + session_bytes // 2, 8) as tight:
        ph = tight.params_create(n, tx, ty)
        s, _ = tight.open_session(ph, pub, w)
        with pytest.raises(dv.DvgpuError) as err:
            tight.open_session(ph, pub, w)
        assert err.value.status == -1 and "HBM budget" in err.value.message
        tight.close_session(s)
        s, _ = tight.open_session(ph, pub, w)  # the footprint was returned
    with dv.DynaverseEngine(1 << 30, 8) as e:
        ph = e.params_create(n, tx, ty)
        with pytest.raises(dv.DvgpuError) as err:
            e.submit(987654321, [4 * n + 1], [1])
        assert err.value.status == -1 and "unknown session" in err.value.message
        s, proof = e.open_session(ph, pub, w)
        ref = D.Session(D.Params(n, tx, ty, "scalar"), pub, w)
        assert proof == ref.proof.to_bytes()
        with pytest.raises(dv.DvgpuError) as err:
            e.params_destroy(ph)
        assert "open sessions" in err.value.message
        # a parameter build holds the engine's worker while an update queues;
        # the close that follows it finds the update pending
        tx2, ty2 = D.sample_trapdoors(15304, 64)
        extra = {}
        busy = threading.Thread(target=lambda: extra.setdefault("p", e.params_create(64, tx2, ty2)))
        busy.start()
        import time
        time.sleep(0.01)
        idx, vals = _mul_edit(n, w, 3, 12345)
        t = e.submit(s, idx, vals)
        with pytest.raises(dv.DvgpuError) as err:
            e.close_session(s)
        assert "pending" in err.value.message
        got, _ = e.wait(t)
        busy.join()
        assert got == ref.update(idx, vals).to_bytes()
        e.close_session(s)
        with pytest.raises(dv.DvgpuError):
            e.close_session(s)
        e.params_destroy(ph)
        e.params_destroy(extra["p"])
        assert e.stats().resident_bytes == 0


@pytest.mark.parametrize("workload", ["hotspot", "spreading"])
def test_reference_benchmark_workloads_n256(engine, workload):
    """The reference's own CPU benchmark sequences (crates/bench/src/bin/
    cpu_dynaverse.rs:240-256) at n = 256, 8 updates: Hotspot adds 1 to s5[0]
    (s4[0] is zero in valid_instance, so the product stays valid); Spreading
    adds 1 to the multiplier of gate 1 + (step - 1) mod (n - 1) and rewrites
    its product.  Every proof against the oracle's."""
    n = 256
    ph, P = _setup(engine, n, 2814 if workload == "hotspot" else 2815)
    pub, w = D.valid_instance(n)
    s, proof = engine.open_session(ph, pub, w)
    ref = D.Session(P, pub, w)
    assert proof == ref.proof.to_bytes()
    for step in range(1, 9):
        cur = ref.current
        if workload == "hotspot":
            idx, vals = [4 * n], [(cur[4 * n] + 1) % R]
        else:
            gate = 1 + (step - 1) % (n - 1)
            mult = (cur[4 * n + gate] + 1) % R
            idx, vals = [4 * n + gate, 5 * n + gate], [mult, cur[3 * n + gate] * mult % R]
        expect = ref.update(idx, vals)
        assert engine.update(s, idx, vals) == expect.to_bytes(), (workload, step)
    engine.close_session(s)
