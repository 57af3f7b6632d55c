"""G1 transform (EC-NTT) parity on the GPU against the oracle's G1 FFT,
which tests/test_oracle_golden.py pins to the DFT definition.  Mirrors the
G1 row transforms of crates/gpu/tests/transform_packet.rs and
stepped_ntt_backend.rs (forward, inverse, round trip, identity rows)."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,rows", [(1, 3), (2, 2), (4, 1), (8, 5), (64, 2), (256, 1), (1024, 1)])
def test_g1_ntt_rows_match_oracle(backend, oracle, n, rows):
    pts, _ = oracle.srs_g1(800 + n, n * rows)
    for inverse in (False, True):
        assert backend.g1_ntt_rows(pts, n, inverse) == oracle.g1_fft(pts, n, inverse), (n, rows, inverse)


def test_g1_ntt_round_trip_identity_and_invalid(backend, oracle, dv):
    n = 512
    pts, _ = oracle.srs_g1(901, 2 * n)
    pts = bytearray(pts)
    pts[64 * 3:64 * 4] = bytes(64)  # infinity entries are valid inputs
    pts = bytes(pts)
    fwd = backend.g1_ntt_rows(pts, n)
    assert backend.g1_ntt_rows(fwd, n, inverse=True) == pts
    zero = bytes(64 * 16)
    assert backend.g1_ntt_rows(zero, 16) == zero
    bad = bytearray(pts[:64 * 8])
    bad[64 * 2 + 1] ^= 1  # off the curve
    with pytest.raises(dv.DvgpuError) as e:
        backend.g1_ntt_rows(bytes(bad), 8)
    assert e.value.status == -1
    with pytest.raises(dv.DvgpuError):
        backend.g1_ntt_rows(pts[:64 * 6], 3)  # not a power of two
    assert backend.g1_ntt_rows(pts[:64 * 4], 4) == oracle.g1_fft(pts[:64 * 4], 4)
