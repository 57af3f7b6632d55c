"""Oracle parity at the full sizes of the operator configurations.

Every output here is compared byte for byte with the CPU oracle on the same
seeded inputs (no round trips or split-sum properties):

* Fr NTT at 2^20, 2^22 and 2^24, forward, inverse, coset forward and coset
  inverse (2^23 and 2^24 take the three-pass schedule), and a batched NTT
  whose largest item is 2^23 (crates/gpu/tests/ntt_backend.rs:133-150 runs
  the reference's full-scale sizes the same way, against arkworks);
* G1 MSM at 2^20 and 2^22 through the plain call and the resident path
  with a table of window multiples (icicle_backend.rs:65-116);
* G2 MSM at 2^16 over [tau^i]G2;
* the batched G2 subgroup check on 2^16 points, half [s]G2 and half twist
  points without cofactor clearing, algorithms 1, 2 and 3
  (g2_validation/tests.rs:24-31);
* sparse MSMs of k = 16, 256 and 4096 entries drawn without replacement
  from 2^16 resident bases (sparse_msm_backend.rs);
* the G1 transform of 16 rows of 2^12 points (transform_packet.rs).

Large inputs are generated on the device (seeded) and copied to the host;
the oracle runs with every host thread, several independent oracle calls
at once (ctypes releases the GIL)."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
KINDS = ["forward", "inverse", "coset_forward", "coset_inverse"]


def _fr_device(torch, backend, seed, n):
    d = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    backend.random_fr_device(seed, n, d.data_ptr())
    return d


def _srs_device(torch, backend, seed, n, g2=False):
    sc = _fr_device(torch, backend, seed, n)
    pts = torch.empty(n * (128 if g2 else 64), dtype=torch.uint8, device="cuda")
    backend.fixed_base_device(sc.data_ptr(), n, g2, pts.data_ptr())
    torch.cuda.synchronize()
    return pts


def _host(t):
    return t.cpu().numpy().tobytes()


@pytest.mark.parametrize("logn", [20, 22, 24])
def test_ntt_full_size_every_kind_matches_oracle(backend, oracle, logn):
    import torch
    n = 1 << logn
    src = _fr_device(torch, backend, 9400 + logn, n)
    vals = _host(src)
    with ThreadPoolExecutor(4) as pool:
        expect = {k: pool.submit(oracle.ntt, vals, k) for k in KINDS}
        out = torch.empty_like(src)
        for kind_id, kind in enumerate(KINDS):
            backend.ntt_device(src.data_ptr(), n, kind_id, out.data_ptr())
            torch.cuda.synchronize()
            assert _host(out) == expect[kind].result(), f"2^{logn} {kind}"
    # the host-buffer entry points over the same input
    if logn == 20:
        assert backend.ntt(vals, inverse=False) == expect["forward"].result()
        assert backend.ntt_coset(vals, inverse=True) == expect["coset_inverse"].result()


def test_ntt_batch_with_a_three_pass_item_matches_oracle(backend, oracle):
    logs = [10, 23, 12, 16]
    kinds = [0, 1, 2, 3]
    vals = [oracle.uniform_fr(9500 + i, 1 << lg) for i, lg in enumerate(logs)]
    got = backend.ntt_batch(b"".join(vals), logs, kinds)
    with ThreadPoolExecutor(4) as pool:
        expect = list(pool.map(lambda a: oracle.ntt(a[0], KINDS[a[1]]), zip(vals, kinds)))
    pos = 0
    for lg, e in zip(logs, expect):
        size = 32 << lg
        assert got[pos:pos + size] == e, f"item 2^{lg}"
        pos += size


@pytest.mark.parametrize("logn", [20, 22])
def test_g1_msm_full_size_matches_oracle(backend, oracle, logn):
    import torch
    n = 1 << logn
    pts = _host(_srs_device(torch, backend, 9600 + logn, n))
    sc = _host(_fr_device(torch, backend, 9700 + logn, n))
    expect = oracle.msm_g1(pts, sc, threads=THREADS)
    assert backend.msm(pts, sc) == expect
    handle = backend.register_bases(pts)
    try:
        assert backend.msm_resident_host(handle, sc) == expect
        backend.precompute_bases(handle, 0)
        assert backend.msm_resident_host(handle, sc) == expect
    finally:
        backend.release_bases(handle)


def test_g2_msm_2_16_matches_oracle(backend, oracle):
    import torch
    n = 1 << 16
    pts = _host(_srs_device(torch, backend, 9800, n, g2=True))
    sc = _host(_fr_device(torch, backend, 9801, n))
    assert backend.msm_g2_host(pts, sc) == oracle.msm_g2(pts, sc, threads=THREADS)


@pytest.mark.parametrize("algorithm", [1, 2, 3])
def test_g2_subgroup_check_2_16_corpus_matches_oracle(backend, oracle, algorithm):
    import torch
    half = 1 << 15
    valid = _srs_device(torch, backend, 9900, half, g2=True)
    twist = torch.empty(half * 128, dtype=torch.uint8, device="cuda")
    backend.random_twist_device(9901, half, twist.data_ptr())
    torch.cuda.synchronize()
    wire = _host(valid) + _host(twist)
    masks, rep = backend.inspect_g2_validation(wire, algorithm)
    expect = oracle.g2_check(wire, algorithm, threads=THREADS)
    assert masks.tolist() == expect.tolist()
    assert (expect[:half] == 0).all() and (expect[half:] == 4).all()
    assert rep.checked_points == 2 * half and rep.invalid_points == half and rep.first_invalid == half


@pytest.mark.parametrize("k", [16, 256, 4096])
def test_sparse_msm_over_2_16_resident_bases_matches_oracle(backend, oracle, k):
    import torch
    n = 1 << 16
    bases = _host(_srs_device(torch, backend, 10000, n))
    rng = np.random.default_rng(10001 + k)
    reqs = []
    for j in range(3):
        idx = rng.choice(n, size=k, replace=False).astype(np.uint64)
        reqs.append((idx, oracle.uniform_fr(10100 + 10 * k + j, k)))
    idx_all = np.concatenate([r[0] for r in reqs])
    vals_all = b"".join(r[1] for r in reqs)
    offs = np.concatenate([[0], np.cumsum([len(r[0]) for r in reqs])])
    expect = [oracle.sparse_msm_g1(bases, idx, vals, threads=THREADS) for idx, vals in reqs]
    h = backend.register_bases(bases)
    try:
        assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect
        backend.precompute_bases(h, 8)
        assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect
        assert backend.msm_sparse_batch([(bases, [(int(i), vals[32 * j:32 * j + 32]) for j, i in enumerate(idx)])
                                         for idx, vals in reqs]) == expect
    finally:
        backend.release_bases(h)


def test_g1_transform_16_rows_of_2_12_matches_oracle(backend, oracle):
    import torch
    n, rows = 1 << 12, 16
    pts = _host(_srs_device(torch, backend, 10200, n * rows))
    for inverse in (False, True):
        assert backend.g1_ntt_rows(pts, n, inverse) == oracle.g1_fft(pts, n, inverse, threads=THREADS), inverse
