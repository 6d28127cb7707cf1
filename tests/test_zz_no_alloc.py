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


def test_noalloc_reads_pinned_tables_before_returning():
    """A caller may hand over pointer tables in pinned memory and reuse them
    as soon as the call returns.  The tables here are pinned; right after the
    call they are overwritten with the addresses of decoy slices while a
    sleep kernel still holds the stream, so a copy of the tables made after
    the return would compute from (and write to) the decoys."""
    import ctypes

    import torch

    import par2gpu

    k, S, r = 96, 4096 + 128, 17
    rng = np.random.default_rng(7)
    src = torch.from_numpy(rng.integers(0, 256, (k, S), dtype=np.uint8)).cuda()
    decoy_src = torch.from_numpy(rng.integers(0, 256, (k, S), dtype=np.uint8)).cuda()
    exps = np.arange(r, dtype=np.uint32)
    want = par2gpu.Context(0)
    ref = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
    want.encode([src[i] for i in range(k)], S, exps, [ref[e] for e in range(r)], device=True)
    want.close()
    got = torch.full((r, S), 0xAB, dtype=torch.uint8, device="cuda")
    decoy_out = torch.full((r, S), 0x5C, dtype=torch.uint8, device="cuda")
    src_tab = torch.tensor([src[i].data_ptr() for i in range(k)], dtype=torch.int64).pin_memory()
    out_tab = torch.tensor([got[e].data_ptr() for e in range(r)], dtype=torch.int64).pin_memory()
    stream = torch.cuda.current_stream()
    torch.cuda._sleep(50_000_000)  # ~25 ms of device time ahead of the call's copies
    par2gpu.check(par2gpu.lib().p2g_encode_noalloc(
        ctypes.c_void_p(stream.cuda_stream), src_tab.data_ptr(), k, S, exps.ctypes.data, r,
        out_tab.data_ptr()))
    src_tab.copy_(torch.tensor([decoy_src[i].data_ptr() for i in range(k)], dtype=torch.int64))
    out_tab.copy_(torch.tensor([decoy_out[e].data_ptr() for e in range(r)], dtype=torch.int64))
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    assert bool((decoy_out == 0x5C).all())


def test_noalloc_leaves_free_device_memory_unchanged():
    """The entry point's promise: once a shape has run (which loads its
    kernels), further calls take no device memory at all."""
    import torch

    import par2gpu

    shapes = [(40, 4096, 5), (300, 16384 + 64, 24), (128, 65536, 40), (2, 64, 1)]
    bufs = []
    for call, (k, S, r) in enumerate(shapes):
        rng = np.random.default_rng(200 + call)
        src = torch.from_numpy(rng.integers(0, 256, (k, S), dtype=np.uint8)).cuda()
        out = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
        bufs.append((src, out, np.arange(r, dtype=np.uint32)))
    stream = torch.cuda.current_stream().cuda_stream

    def run_all():
        for src, out, exps in bufs:
            par2gpu.encode_noalloc(stream, [s for s in src], src.shape[1], exps,
                                   [o for o in out])
        torch.cuda.synchronize()

    run_all()  # loads every kernel the shapes use
    first = [o.clone() for _, o, _ in bufs]
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        run_all()
    assert torch.cuda.mem_get_info()[0] == free0
    for (_, out, _), f in zip(bufs, first):
        assert torch.equal(out, f)
