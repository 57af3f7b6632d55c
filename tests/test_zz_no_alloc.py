"""The allocation-free NTT entry point (dvgpu_bn254_ntt_noalloc).

It exists for callers that cannot allocate device memory when they need a
transform (an allocator or memory pool owns device memory, a latency-critical
path must not synchronise on cudaMalloc/cudaFree, or a fixed device-memory
budget).  Its scratch is one static device array shared by every call, so
this test checks, through the C-ABI, that two calls in a row give exactly the
output of the ordinary device entry point (dvgpu_bn254_ntt_device), for every
transform kind and for sizes up to the 65536-element limit, and that a larger
size is rejected.  The file is named so pytest collects it last.
"""
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_ntt_matches_device_entry_point_on_consecutive_calls(dv):
    import torch

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    with dv.DvgpuBackend() as b:
        for logn in (0, 1, 3, 10, 13, 16):
            n = 1 << logn
            src = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
            b.random_fr_device(9100 + logn, n, src.data_ptr(), s)
            for kind in (0, 1, 2, 3):
                ref = torch.empty_like(src)
                b.ntt_device(src.data_ptr(), n, kind, ref.data_ptr(), s)
                expect = ref.cpu()
                for _ in range(2):  # the shared scratch keeps the previous call's contents
                    out = torch.full_like(src, 0xAB)
                    dv.ntt_noalloc(src.data_ptr(), n, kind, out.data_ptr(), s)
                    assert torch.equal(out.cpu(), expect), f"n={n} kind={kind}"
        big = torch.empty((1 << 17) * 32, dtype=torch.uint8, device="cuda")
        with pytest.raises(dv.DvgpuError) as e:
            dv.ntt_noalloc(big.data_ptr(), 1 << 17, 0, big.data_ptr(), s)
        assert e.value.status == -1 and "65536" in e.value.message
