"""The update-proof benchmark's inputs and its CPU baseline (no GPU).

The stream must be one the reference's session accepts: every update is a
set of circuit-valid multiplication-gate edits (toy_circuit.rs:72-90), the
supports follow the stated distribution, and the trapdoors pass the setup's
rejection rules (srs.rs:158-178).  The CPU baseline runs the oracle's
restatement of the reference's steps on the benchmark's own requests."""
import bench
from oracle import dynaverse as D

R = D.R


def test_trapdoors_pass_the_setup_rules():
    for n, (tx, ty) in bench.bench_trapdoors([16, 256, 4096]).items():
        m = 8 * n
        assert 0 < tx < R and 0 < ty < R and tx != ty
        assert pow(tx, m, R) != 1 and pow(ty, m, R) != 1 and tx != pow(ty, 8, R)


def test_stream_updates_keep_every_gate_valid():
    sizes = [16, 16, 256]
    wit = {n: bench.valid_witness(n, 9000 + n.bit_length()) for n in set(sizes)}
    cur = {j: list(wit[n][1]) for j, n in enumerate(sizes)}
    reqs = bench.proof_stream(sizes, [wit[n][1] for n in sizes], 80, 5.0, 9100)
    wide = 0
    for t, (j, idx, vals) in enumerate(reqs):
        n = sizes[j]
        values = [int.from_bytes(vals[32 * i:32 * i + 32], "little") for i in range(len(idx))]
        assert len(idx) % 2 == 0 and 2 <= len(idx) <= 2 * min(n, 32)
        gates = sorted({i % n for i in idx})
        assert all(4 * n <= i < 6 * n for i in idx) and len(gates) == len(idx) // 2
        for i, v in zip(idx, values):
            cur[j][i] = v
        assert D.check_gates(n, wit[n][0], cur[j], gates) is None
        span = max(gates) - min(gates)
        if t % 2:
            assert span < 64  # the session's hotspot window
        else:
            wide += span >= 64
    assert wide  # uniform supports spread past the window


def test_cpu_baseline_runs_the_benchmark_requests():
    class Args:
        log_n, sessions, mix, requests, umax = 4, 3, False, 12, 3.0
    op = bench.ProofServeOp(Args)
    op._inputs()
    cpu = bench.ProofsCpu(op, threads=2)
    rate = cpu.sample(60.0)
    assert cpu.pos == len(op.reqs)  # every request applied, none rejected
    assert cpu.count + cpu.rebuilds == len(op.reqs)
    assert rate is None or rate > 0
    assert "the benchmark's own request stream" in cpu.describe()
