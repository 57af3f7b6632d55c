"""Batching parity on the GPU: the batched NTT (one persistent launch for
transforms of uneven sizes) and CUDA-graph batch plans (uneven G1 MSMs over
prefixes of resident bases plus NTTs), each compared with the oracle and
with the plain per-call entry points on the same inputs.

The reference batches MSMs with next-pow2 padding and 64-set groups
(crates/gpu/src/icicle.rs:281-339, native/src/icicle_msm.cu:810-880) and
runs NTTs one call per vector (icicle.rs:429-456); its tests compare every
batched result with arkworks (crates/gpu/tests/icicle_backend.rs:131-189).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KINDS = ["forward", "inverse", "coset_forward", "coset_inverse"]


class _DeviceBytes:
    """Wraps a raw device pointer for torch.as_tensor."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3}


def _device_view(ptr, nbytes):
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


def _split(buf, logs):
    out, off = [], 0
    for L in logs:
        n = 32 << L
        out.append(buf[off:off + n])
        off += n
    return out


def test_ntt_batch_uneven_sizes_match_oracle(backend, oracle):
    logs = [1, 2, 3, 5, 8, 10, 11, 12, 13, 7, 14, 16, 4, 11, 12]
    kinds = [i % 4 for i in range(len(logs))]
    parts = [oracle.uniform_fr(9100 + i, 1 << L) for i, L in enumerate(logs)]
    got = _split(backend.ntt_batch(b"".join(parts), logs, kinds), logs)
    for i, (L, k) in enumerate(zip(logs, kinds)):
        assert got[i] == oracle.ntt(parts[i], KINDS[k]), f"transform {i}: 2^{L} {KINDS[k]}"
    # all forward (kinds omitted) and a single transform
    fwd = _split(backend.ntt_batch(b"".join(parts[:4]), logs[:4]), logs[:4])
    for i in range(4):
        assert fwd[i] == oracle.ntt(parts[i], "forward")
    assert backend.ntt_batch(parts[11], [16], [1]) == oracle.ntt(parts[11], "inverse")


def test_ntt_batch_device_matches_per_call(backend, oracle):
    import torch
    logs = [20, 10, 15, 18, 12, 19, 11, 16]
    kinds = [0, 1, 2, 3, 0, 1, 2, 3]
    total = sum(1 << L for L in logs)
    d_in = torch.empty(total * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(4242, total, d_in.data_ptr())
    d_out = torch.empty_like(d_in)
    backend.ntt_batch_device(d_in.data_ptr(), logs, d_out.data_ptr(), kinds)
    ref = torch.empty_like(d_in)
    off = 0
    for L, k in zip(logs, kinds):
        n = 1 << L
        backend.ntt_device(d_in.data_ptr() + 32 * off, n, k, ref.data_ptr() + 32 * off)
        off += n
    torch.cuda.synchronize()
    assert torch.equal(d_out, ref)
    # round trip through the batch: inverse of the forward batch
    fwd_logs = [20, 12, 17]
    tot2 = sum(1 << L for L in fwd_logs)
    x = d_in[:tot2 * 32].clone()
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    torch.cuda.synchronize()
    backend.ntt_batch_device(x.data_ptr(), fwd_logs, y.data_ptr(), [2, 0, 2])
    backend.ntt_batch_device(y.data_ptr(), fwd_logs, z.data_ptr(), [3, 1, 3])
    torch.cuda.synchronize()
    assert torch.equal(x, z)


def test_ntt_batch_rejects_bad_input(backend, oracle, dv):
    logs = [4, 6, 5]
    parts = [oracle.uniform_fr(9300 + i, 1 << L) for i, L in enumerate(logs)]
    bad = bytearray(parts[1])
    bad[32 * 7:32 * 8] = b"\xff" * 32
    with pytest.raises(dv.DvgpuError) as e:
        backend.ntt_batch(parts[0] + bytes(bad) + parts[2], logs)
    assert e.value.status == -1 and "transform 1" in e.value.message
    for bad_log in (0, 25):
        with pytest.raises(dv.DvgpuError):
            backend.ntt_batch(bytes(32 * 16), [bad_log])
    with pytest.raises(dv.DvgpuError):
        backend.ntt_batch(parts[0], [4], [7])
    # the owner stays healthy
    assert backend.ntt_batch(parts[0], [4]) == oracle.ntt(parts[0], "forward")


def _plan_sizes(seed, nbases, count):
    rng = np.random.default_rng(seed)
    sizes = [int(min(nbases, max(1, round(2 ** rng.uniform(0, np.log2(nbases)))))) for _ in range(count)]
    sizes[0] = 1
    sizes[1] = nbases
    return sizes


def test_batch_plan_matches_oracle_and_replays(backend, oracle, dv):
    nbases = 4096
    pts, _ = oracle.srs_g1(5150, nbases)
    sizes = _plan_sizes(5151, nbases, 40)
    logs = [3, 10, 12, 13, 1, 11]
    kinds = [0, 1, 2, 3, 0, 1]
    h = backend.register_bases(pts)
    try:
        plan, log = backend.batch_plan_create(h, sizes, logs, kinds)
        assert len(log["classes"]) >= 4 and log["graph_nodes"] > 0
        assert sum(c["sets"] for c in log["classes"]) == len(sizes)
        for c in log["classes"]:
            assert c["best_c"] in [x["c"] for x in c["candidates"]]
            # bucket partition: the reduction's segment length, tried around the rule's
            assert c["best_seg"] in [x["seg"] for x in c["seg_candidates"]]
        # the NTT's tile (2^10..2^12 elements) and register round (radix 2,
        # 4, 8) are picked from every pair, each checked against the first
        # on the device while the plan is built
        pairs = [(x["tile"], x["radix"]) for x in log["ntt"]["candidates"]]
        assert pairs == [(t, r) for t in (1024, 2048, 4096) for r in (2, 4, 8)]
        assert (log["ntt"]["best_tile"], log["ntt"]["best_radix"]) in pairs
        for rep in range(2):  # the second run replays the graph on new inputs
            scs = [oracle.uniform_fr(5200 + 100 * rep + i, n) for i, n in enumerate(sizes)]
            scs[3] = bytes(32 * sizes[3])  # all-zero scalars: infinity
            vals = [oracle.uniform_fr(5300 + 100 * rep + j, 1 << L) for j, L in enumerate(logs)]
            msm, ntt = backend.batch_plan_run(plan, b"".join(scs), b"".join(vals), len(sizes))
            for i, n in enumerate(sizes):
                assert msm[i] == oracle.msm_g1(pts[:64 * n], scs[i]), f"rep {rep} MSM {i} (n={n})"
            assert msm[3] == bytes(64)
            for j, part in enumerate(_split(ntt, logs)):
                assert part == oracle.ntt(vals[j], KINDS[kinds[j]]), f"rep {rep} NTT {j}"
        # host-buffer runs check every input before writing any output: a bad
        # scalar or NTT value fails the call, the output buffers stay as they
        # were, and the plan runs again afterwards
        total = sum(sizes)
        nvals = sum(1 << L for L in logs)
        lib = dv.lib()
        for bad_scalar in (True, False):
            sc = bytearray(b"".join(scs))
            vv = bytearray(b"".join(vals))
            if bad_scalar:
                sc[32 * (total - 5):32 * (total - 4)] = b"\xff" * 32
            else:
                vv[32 * (nvals - 3):32 * (nvals - 2)] = b"\xff" * 32
            mo = ctypes.create_string_buffer(b"\xab" * (64 * len(sizes)), 64 * len(sizes))
            no = ctypes.create_string_buffer(b"\xcd" * (32 * nvals), 32 * nvals)
            err = ctypes.create_string_buffer(256)
            rc = lib.dvgpu_batch_plan_run(backend.handle, plan, bytes(sc), bytes(vv), mo, no, err, 256)
            assert rc == -1 and b"non-canonical" in err.value
            assert mo.raw == b"\xab" * (64 * len(sizes)) and no.raw == b"\xcd" * (32 * nvals)
        msm, ntt = backend.batch_plan_run(plan, b"".join(scs), b"".join(vals), len(sizes))
        assert msm[0] == oracle.msm_g1(pts[:64 * sizes[0]], scs[0])
        assert _split(ntt, logs)[1] == oracle.ntt(vals[1], KINDS[kinds[1]])
        backend.batch_plan_destroy(plan)
    finally:
        backend.release_bases(h)


def test_batch_plan_device_buffers_match_per_call(backend, oracle, dv):
    import torch
    nbases = 1 << 15
    pts, _ = oracle.srs_g1(6150, nbases)
    sizes = _plan_sizes(6151, nbases, 64)
    logs = [16, 11, 14, 9]
    h = backend.register_bases(pts)
    try:
        plan, _ = backend.batch_plan_create(h, sizes, logs)
        buf = backend.batch_plan_buffers(plan)
        assert buf.scalar_bytes == 32 * sum(sizes) and buf.msm_result_bytes == 64 * len(sizes)
        backend.random_fr_device(61, sum(sizes), buf.scalars)
        backend.random_fr_device(62, sum(1 << L for L in logs), buf.ntt_values)
        torch.cuda.synchronize()
        for _ in range(3):
            backend.batch_plan_launch(plan)
        backend.batch_plan_check(plan)
        msm = _device_view(buf.msm_results, buf.msm_result_bytes).cpu().numpy().tobytes()
        ntt = _device_view(buf.ntt_results, buf.ntt_bytes).cpu()
        off = 0
        for i, n in enumerate(sizes):
            got = msm[64 * i:64 * (i + 1)]
            assert got == backend.msm_resident(h, buf.scalars + 32 * off, n), f"MSM {i} (n={n})"
            off += n
        ref = torch.empty(buf.ntt_bytes, dtype=torch.uint8, device="cuda")
        off = 0
        for L in logs:
            backend.ntt_device(buf.ntt_values + 32 * off, 1 << L, 0, ref.data_ptr() + 32 * off)
            off += 1 << L
        torch.cuda.synchronize()
        assert torch.equal(ntt, ref.cpu())
        # a non-canonical scalar is reported by check (-1) and the owner stays healthy
        _device_view(buf.scalars + 32 * 5, 32).fill_(255)
        torch.cuda.synchronize()
        backend.batch_plan_launch(plan)
        with pytest.raises(dv.DvgpuError) as e:
            backend.batch_plan_check(plan)
        assert e.value.status == -1 and "index 5" in e.value.message
        backend.batch_plan_destroy(plan)
        with pytest.raises(dv.DvgpuError):
            backend.batch_plan_launch(plan)
    finally:
        backend.release_bases(h)


def test_batch_plan_ntt_only_and_invalid_arguments(backend, oracle, dv):
    plan, log = backend.batch_plan_create(0, [], [5, 12], [1, 2])
    vals = [oracle.uniform_fr(7300 + j, 1 << L) for j, L in enumerate([5, 12])]
    _, ntt = backend.batch_plan_run(plan, None, b"".join(vals), 0)
    parts = _split(ntt, [5, 12])
    assert parts[0] == oracle.ntt(vals[0], "inverse") and parts[1] == oracle.ntt(vals[1], "coset_forward")
    backend.batch_plan_destroy(plan)
    pts, _ = oracle.srs_g1(7350, 64)
    h = backend.register_bases(pts)
    try:
        with pytest.raises(dv.DvgpuError):
            backend.batch_plan_create(h, [65], [])  # beyond the registered bases
        with pytest.raises(dv.DvgpuError):
            backend.batch_plan_create(h, [0], [])
        with pytest.raises(dv.DvgpuError):
            backend.batch_plan_create(h + 999, [4], [])
        with pytest.raises(dv.DvgpuError):
            backend.batch_plan_create(h, [], [25])
    finally:
        backend.release_bases(h)
