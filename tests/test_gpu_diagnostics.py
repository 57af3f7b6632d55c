"""Diagnostic entry points the reference's Rust crate binds beside the
compute path: the MSM phase timeline (crates/gpu/src/icicle.rs:54,250),
the G2 check kernel configuration, resources and experiment counters
(crates/gpu/src/g2_validation.rs:91-94) and the profiled resident call
(crates/gpu/src/resident_profile.rs:40).  Each must leave results identical
to the plain calls."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_msm_timeline_matches_plain_msm(backend, oracle):
    n = 3000
    points = oracle.fixed_base_g1(oracle.uniform_fr(7101, n))
    scalars = oracle.uniform_fr(7102, n)
    res, tm, tl = backend.msm_with_timeline(points, scalars)
    assert res == oracle.msm_g1(points, scalars) == backend.msm(points, scalars)
    assert tl.bitsize == 254 and tl.c >= 1 and tl.windows == (255 + tl.c - 1) // tl.c
    assert tl.buckets == tl.windows << (tl.c - 1)
    assert list(tl.bytes)[1:3] == [64 * n, 32 * n] and tl.bytes[5] == 64 and tl.bytes[7] == 4
    assert all(tl.calls[k] == 1 for k in (0, 1, 2, 3, 4, 5, 7)) and tl.calls[8] == 0
    assert tl.event_ns[3] > 0 and tl.kernel_ns[6] > 0 and tl.kernel_calls[6] == 1
    assert tl.instrumentation_inclusive_ns >= tl.wall_ns[3] and tm.icicle_ns > 0
    empty, _, tl0 = backend.msm_with_timeline(b"", b"")
    assert empty == bytes(64) and tl0.bitsize == 254 and tl0.calls[3] == 0


def test_g2_kernel_config_resources_and_counters(backend, oracle, dv):
    one = (1).to_bytes(32, "little")
    good = oracle.fixed_base_g2(oracle.uniform_fr(7201, 200) + one)
    wire = bytearray(good)
    wire[128 * 7 + 5] ^= 1                       # off the curve
    wire = bytes(wire)
    default = backend.g2_kernel_config()
    assert (default.threads, default.schedule, default.layout, default.fused) == (128, 0, 0, 0)
    base_masks, base_rep = backend.inspect_g2_validation(wire, 3)
    assert base_rep.invalid_points >= 1 and base_masks[7] != 0
    before = backend.g2_experiment_stats().subgroup_kernel_ns
    try:
        for threads in (64, 256, 128):
            backend.g2_kernel_config((threads, 1, 1, 1))
            masks, rep = backend.inspect_g2_validation(wire, 3)
            assert list(masks) == list(base_masks) and rep.invalid_points == base_rep.invalid_points
            r = backend.g2_kernel_resources(3)
            assert r.block_threads == threads and r.registers > 0 and r.active_blocks >= 1
            assert r.max_threads_per_sm >= threads and r.normalize_registers > 0
        st = backend.g2_experiment_stats()
        assert st.subgroup_kernel_ns > before and st.repack_device_ns == 0 and st.logical_repack_bytes == 0
        for bad in ((96, 0, 0, 0), (128, 2, 0, 0), (128, 0, 2, 0), (128, 0, 0, 2)):
            with pytest.raises(dv.DvgpuError):
                backend.g2_kernel_config(bad)
        assert backend.g2_kernel_config().threads == 128
        with pytest.raises(dv.DvgpuError):
            backend.g2_kernel_resources(4)
    finally:
        backend.g2_kernel_config((128, 0, 0, 0))


def test_resident_call_profiled_matches_plain_call(dv, oracle):
    b = dv.DvgpuBackend()
    try:
        root = pow(5, (0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001 - 1) >> 20,
                   0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001)
        b.resident_configure(1 << 28, 64 * 144, root.to_bytes(32, "little"))
        h, prof = b.resident_call_profiled("ALLOC", kind=0, length=32, flags=1)
        assert b.rb_len(h) == 32 and prof.native_wall_ns > 0 and prof.event_mask == 4
        vals = oracle.uniform_fr(7301, 32)
        buf = ctypes.create_string_buffer(vals, len(vals))
        _, prof = b.resident_call_profiled("WRITE", kind=0, a=h, a_offset=0, length=32,
                                           input=ctypes.addressof(buf))
        assert prof.h2d_bytes == 32 * 32 and prof.d2h_bytes == 0
        assert prof.native_wall_ns >= prof.operation_host_ns
        out = ctypes.create_string_buffer(32 * 32)
        _, prof = b.resident_call_profiled("READ", kind=0, a=h, a_offset=0, length=32,
                                           output=ctypes.addressof(out))
        assert out.raw == vals == b.rb_read(h, 0, 32, 0) and prof.d2h_bytes == 32 * 32
        with pytest.raises(dv.DvgpuError):
            b.resident_call_profiled("READ", kind=0, a=h, a_offset=30, length=8, output=ctypes.addressof(out))
    finally:
        b.close()
