"""Concurrent calls through the C ABI.

The reference calls its strategy from every rayon worker at once
(`par2_rs.rs:859-864` from `StreamingEncoder::flush_batch`, `:588-599` from
`reconstruct_streaming_chunk`), so the library must be thread-safe and
reentrant: one shared context serialises its own calls, separate contexts
run side by side, and `p2g_last_error` is per thread.  ctypes releases the
GIL for the duration of each call, so these threads really do overlap in the
library.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

THREADS = 8


def _work(seed):
    """One worker's inputs and the oracle's answers for them."""
    rng = np.random.default_rng(seed)
    k, S, r = 20 + seed, 2048 + 2 * seed, 3 + seed % 5
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = rng.choice(1000, r, replace=False).astype(np.uint32)
    data = rng.integers(0, 65536, 777, dtype=np.uint16)
    dst = rng.integers(0, 65536, 777, dtype=np.uint16)
    c = int(rng.integers(1, 65536))
    want_mac = dst ^ np.array([oracle.gf_mul(int(v), c) for v in data], np.uint16)
    return src, exps, oracle.encode(src, exps), data, dst, c, want_mac


def _run(ctx, w):
    src, exps, want_enc, data, dst, c, want_mac = w
    for _ in range(3):
        got = ctx.encode_array(src, exps)
        if not np.array_equal(got, want_enc):
            return "encode differs"
        d = dst.copy()
        ctx.muladd(d, data, c)
        if not np.array_equal(d, want_mac):
            return "muladd differs"
    return None


def test_shared_context_from_many_threads():
    import par2gpu

    works = [_work(s) for s in range(THREADS)]
    with par2gpu.Context(0) as ctx:
        with ThreadPoolExecutor(THREADS) as ex:
            errs = list(ex.map(lambda w: _run(ctx, w), works))
    assert errs == [None] * THREADS


def test_context_per_thread():
    import par2gpu

    works = [_work(100 + s) for s in range(THREADS)]

    def one(w):
        with par2gpu.Context(0) as ctx:
            return _run(ctx, w)

    with ThreadPoolExecutor(THREADS) as ex:
        errs = list(ex.map(one, works))
    assert errs == [None] * THREADS


def test_last_error_is_per_thread():
    """A failing call on one thread sets that thread's message only; the
    other threads' successful calls clear and keep their own."""
    import par2gpu

    with par2gpu.Context(0) as ctx:
        def bad(_):
            x = np.zeros(7, np.uint8)
            try:
                ctx.encode([x, x], 7, [0], [np.zeros(7, np.uint8)])
            except par2gpu.Par2GpuError as e:
                return e.code, par2gpu.last_error()
            return None, ""

        def good(_):
            src = np.ones((4, 64), np.uint8)
            ctx.encode_array(src, [0, 1])
            return par2gpu.last_error()

        with ThreadPoolExecutor(THREADS) as ex:
            fb = [ex.submit(bad, i) for i in range(THREADS // 2)]
            fg = [ex.submit(good, i) for i in range(THREADS // 2)]
            for f in fb:
                code, msg = f.result()
                assert code == par2gpu.EINVAL and "even" in msg
            for f in fg:
                assert f.result() == ""
