"""GPU parity of the strategy interface's shuffle2x hooks (galois/simd/mod.rs:
68-127) as this library serves them -- device copies of prepared buffers,
multiply-accumulates recorded and run in batches, results written back by
finish -- and of par2-rs's streaming encoder restated over them
(par2_rs.rs:687-902, through p2f_streaming_encode), against the oracle."""
import numpy as np
import pytest

from oracle import oracle
from tests import quickpar

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import par2gpu

    c = par2gpu.Context(0)
    yield c
    c.close()


def u16(rng, *shape):
    return rng.integers(0, 65536, shape, dtype=np.uint16)


def muladd_ref(dst, src, c):
    """dst ^= c * src over u16 symbols, by the oracle."""
    out = dst.copy()
    oracle.muladd_region([out], [src], np.array([[c]], np.uint16), 0, len(out))
    return out


def test_recorded_products_match_oracle(ctx):
    """Accumulators and sources prepared, many products recorded (the same
    pair twice, zero coefficients, a source reused after its buffer was
    re-prepared with new data), one finish per accumulator."""
    rng = np.random.default_rng(1)
    n = 4096 + 24
    accs = [u16(rng, n) for _ in range(5)]
    want = [a.copy() for a in accs]
    for a in accs:
        ctx.prepare_shuffle2x(a)
    batch = [np.zeros(n, np.uint16) for _ in range(3)]
    for rnd in range(4):
        blocks = [u16(rng, n) for _ in batch]
        for b, blk in zip(batch, blocks):
            b[:] = blk                     # a reused batch buffer, new contents
            ctx.prepare_shuffle2x(b)
        for j, a in enumerate(accs):
            for b, blk in zip(batch, blocks):
                for c in (int(rng.integers(0, 65536)), 0, int(rng.integers(1, 65536))):
                    ctx.muladd_shuffle2x(a, b, c)
                    want[j] = muladd_ref(want[j], blk, c)
    for a in accs:
        ctx.finish_shuffle2x(a)
    for a, w in zip(accs, want):
        assert np.array_equal(a, w)


def test_regions_unprepared_buffers_and_finish_without_prepare(ctx):
    rng = np.random.default_rng(2)
    n = 8192
    accs = [u16(rng, n) for _ in range(3)]
    srcs = [u16(rng, n) for _ in range(4)]
    want = [a.copy() for a in accs]
    for a in accs:
        ctx.prepare_shuffle2x(a)
    for s in srcs[:3]:                      # srcs[3] stays unprepared
        ctx.prepare_shuffle2x(s)
    for off, ln in ((0, 2048), (2048, 1000), (3051, 777), (4096, 4096)):   # aligned and not
        co = rng.integers(0, 65536, (3, 4), dtype=np.uint16)
        ctx.muladd_region_shuffle2x(accs, srcs, co, off, ln)
        oracle.muladd_region(want, srcs, co, off, ln)
    # an unprepared destination runs at once, reading a prepared source's data
    plain = u16(rng, n)
    ref = muladd_ref(plain, srcs[0], 777)
    ctx.muladd_shuffle2x(plain, srcs[0], 777)
    assert np.array_equal(plain, ref)
    # a prepared accumulator as the source of an unprepared destination: its
    # recorded products are run and its current value read back
    plain2 = u16(rng, n)
    want2 = muladd_ref(plain2, want[0], 3)
    ctx.muladd_shuffle2x(plain2, accs[0], 3)
    assert np.array_equal(plain2, want2)
    for a in accs:
        ctx.finish_shuffle2x(a)
    for a, w in zip(accs, want):
        assert np.array_equal(a, w)
    never = u16(rng, 64)
    keep = never.copy()
    ctx.finish_shuffle2x(never)             # never prepared: left as it is
    assert np.array_equal(never, keep)


def test_unprepared_destination_reads_accumulated_source(ctx):
    rng = np.random.default_rng(3)
    n = 2048
    acc = u16(rng, n)
    src = u16(rng, n)
    acc_val = muladd_ref(acc, src, 99)
    ctx.prepare_shuffle2x(acc)
    ctx.prepare_shuffle2x(src)
    ctx.muladd_shuffle2x(acc, src, 99)      # recorded: acc's host copy is now stale
    plain = u16(rng, n)
    want = muladd_ref(plain, acc_val, 5)
    ctx.muladd_shuffle2x(plain, acc, 5)     # must see acc after the recorded product
    assert np.array_equal(plain, want)
    ctx.finish_shuffle2x(acc)
    assert np.array_equal(acc, acc_val)


def test_streaming_encoder_quickpar():
    """All 60 recovery slices of the QuickPar set through the restated
    streaming encoder over the CUDA strategy (4 worker threads)."""
    from par2gpu import format as fmt

    qp = quickpar.load()
    src, _ = qp.slices()
    got = fmt.streaming_encode(src, 60, threads=4)
    for e in range(60):
        assert np.array_equal(got[e], qp.recovery[e]), e


@pytest.mark.parametrize("k,S,r,threads", [(1, 64, 1, 1), (37, 4098, 13, 3), (300, 8192, 60, 8),
                                           (129, 65536, 205, 16),
                                           # ragged blocks above 256 KiB: staging copies in parts
                                           (64, (1 << 20) + 6, 9, 8)])
def test_streaming_encoder_matches_oracle(k, S, r, threads):
    from par2gpu import format as fmt

    rng = np.random.default_rng(k + r)
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    want = oracle.encode(src, np.arange(r, dtype=np.uint32))
    assert np.array_equal(fmt.streaming_encode(src, r, threads=threads), want)


def test_streaming_encoder_large_set_with_flushes():
    """1024 x 1 MiB, r = 205: the recorded work crosses the launch threshold
    several times while batches of 128 blocks stream in from 16 threads;
    equal to the restated AVX2 strategy."""
    from par2gpu import format as fmt

    rng = np.random.default_rng(5)
    k, S, r = 1024, 1 << 20, 205
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    got = fmt.streaming_encode(src, r, threads=16)
    assert np.array_equal(got, oracle.cpu_encode(src, r, 16))
