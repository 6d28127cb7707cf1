"""p2g_encode_noalloc: recovery-slice creation for callers that cannot
allocate device memory when they encode (services holding a fixed,
pre-reserved memory budget; latency paths that cannot take cudaMalloc's
implicit synchronisation).  Its scratch is a fixed static device array, so
its results must equal those of the allocating entry point p2g_encode bit for
bit, call after call, whatever the previous call left in that array.

The file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.  It passes alone in a fresh
process and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_equals_encode_on_consecutive_calls():
    import torch

    import par2gpu

    ctx = par2gpu.Context(0)
    stream = torch.cuda.current_stream()
    # two calls in a row with different shapes and contents: the second must
    # not see anything of the first in the shared scratch array
    for call, (k, S, r) in enumerate([(64, 8192, 13), (150, 2048 * 9 + 64, 29)]):
        rng = np.random.default_rng(100 + call)
        src = torch.from_numpy(rng.integers(0, 256, (k, S), dtype=np.uint8)).cuda()
        exps = np.arange(r, dtype=np.uint32)
        want = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
        ctx.encode([src[i] for i in range(k)], S, exps, [want[e] for e in range(r)], device=True)
        got = torch.full((r, S), 0xAB, dtype=torch.uint8, device="cuda")
        par2gpu.encode_noalloc(stream.cuda_stream, [src[i] for i in range(k)], S, exps,
                               [got[e] for e in range(r)])
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}"
    ctx.close()


def test_noalloc_rejects_oversize_problems():
    import torch

    import par2gpu

    src = torch.zeros((2, 64), dtype=torch.uint8, device="cuda")
    out = torch.zeros((1, 64), dtype=torch.uint8, device="cuda")
    # 1100 inputs of 64 KiB need about 70 MB of bit planes: beyond the 64 MiB array
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        par2gpu.encode_noalloc(0, [src[0]] * 1100, 65536, [0], [out[0]])
    assert ei.value.code == par2gpu.ERANGE
    assert "static maximum" in par2gpu.last_error()
