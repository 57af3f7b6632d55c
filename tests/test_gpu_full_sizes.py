"""Size-independent properties at the operator configurations' full sizes,
where the oracle would take too long: an MSM equals the sum of the MSMs of
its two halves and is the same through the plain and the precomputed-table
paths (different window widths and bucket sets); an NTT followed by its
inverse (plain and coset) returns the input; fixed-base outputs agree with
the oracle on a sample.  A 2^23 NTT (three passes) is also compared byte
for byte with the oracle's transform, all four kinds, so an error that the
inverse would undo is caught too.  Inputs are seeded and generated on the
device."""
from concurrent.futures import ThreadPoolExecutor

import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(torch, backend, n, seed):
    sc = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(seed, n, sc.data_ptr())
    pts = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    backend.fixed_base_device(sc.data_ptr(), n, False, pts.data_ptr())
    backend.random_fr_device(seed + 1, n, sc.data_ptr())
    torch.cuda.synchronize()
    return pts.cpu().numpy().tobytes(), sc.cpu().numpy().tobytes()


@pytest.mark.parametrize("logn", [20, 22])
def test_msm_full_size_split_and_paths(backend, oracle, logn):
    import torch
    n = 1 << logn
    pts, sc = _device_inputs(torch, backend, n, 9100 + logn)
    whole = backend.msm(pts, sc)
    h = n // 2
    halves = oracle.g1_add(backend.msm(pts[:64 * h], sc[:32 * h]), backend.msm(pts[64 * h:], sc[32 * h:]))
    assert whole == halves
    handle = backend.register_bases(pts)
    try:
        backend.precompute_bases(handle, 0)
        assert backend.msm_resident_host(handle, sc) == whole
    finally:
        backend.release_bases(handle)


def test_ntt_2_24_round_trips(backend):
    import torch
    n = 1 << 24
    src = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(9200, n, src.data_ptr())
    fwd = torch.empty_like(src)
    back = torch.empty_like(src)
    for f, i in ((0, 1), (2, 3)):  # forward / inverse, coset forward / coset inverse
        backend.ntt_device(src.data_ptr(), n, f, fwd.data_ptr())
        backend.ntt_device(fwd.data_ptr(), n, i, back.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(back, src), (f, i)
        assert not torch.equal(fwd, src)


NTT_KINDS = ["forward", "inverse", "coset_forward", "coset_inverse"]


def test_ntt_2_23_matches_oracle(backend, oracle):
    """2^23 takes three passes of unequal depth (8, 8 and 7 stages); 2^24
    and the batch form are compared in test_gpu_config_parity.py.  The
    oracle's four transforms run at once on the host cores (the ctypes
    calls release the GIL) while the device computes its own."""
    import torch
    n = 1 << 23
    src = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(9323, n, src.data_ptr())
    torch.cuda.synchronize()
    host = src.cpu().numpy().tobytes()
    out = torch.empty_like(src)
    with ThreadPoolExecutor(4) as pool:
        want = [pool.submit(oracle.ntt, host, kind) for kind in NTT_KINDS]
        for k, kind in enumerate(NTT_KINDS):
            backend.ntt_device(src.data_ptr(), n, k, out.data_ptr())
            torch.cuda.synchronize()
            assert out.cpu().numpy().tobytes() == want[k].result(), kind


def test_fixed_base_2_20_sample_matches_oracle(backend, oracle):
    import torch
    n = 1 << 20
    sc = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(9300, n, sc.data_ptr())
    out = torch.empty(n * 64, dtype=torch.uint8, device="cuda")
    backend.fixed_base_device(sc.data_ptr(), n, False, out.data_ptr())
    torch.cuda.synchronize()
    scb, outb = sc.cpu().numpy().tobytes(), out.cpu().numpy().tobytes()
    picks = [0, 1, n // 3, n // 2, n - 2, n - 1] + list(range(4097, 4097 + 58))
    sample = b"".join(scb[32 * i:32 * i + 32] for i in picks)
    expect = oracle.fixed_base_g1(sample)
    assert b"".join(outb[64 * i:64 * i + 64] for i in picks) == expect
