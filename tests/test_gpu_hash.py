"""GPU parity of per-slice MD5 + CRC32 (K3) through the C ABI: the known
answers of par2-rs src/hash/mod.rs:33-67, the QuickPar IFSC entries, ragged
sizes around the MD5 padding boundary, and the CRC-then-MD5 verdict of
verify.rs:610-648."""
import hashlib
import zlib

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


def one(ctx, data):
    a = np.frombuffer(data, np.uint8).copy() if len(data) else np.zeros(0, np.uint8)
    md5, crc = ctx.hash_slices([a], len(data))
    return md5[0].tobytes().hex(), int(crc[0])


def test_known_answers(ctx):
    assert one(ctx, b"") == ("d41d8cd98f00b204e9800998ecf8427e", 0)
    assert one(ctx, b"abc") == ("900150983cd24fb0d6963f7d28e17f72", 0x352441C2)
    assert one(ctx, b"message digest")[0] == "f96b697d7cb7938d525a2f31aaf161d0"
    msg = b"12345678901234567890123456789012345678901234567890123456789012345678901234567890"
    assert one(ctx, msg)[0] == "57edf4a22be3c955ac49da2e2107b67a"


def test_ragged_sizes(ctx):
    rng = np.random.default_rng(3)
    for n in list(range(0, 130)) + [511, 512, 1000, 4095, 4096, 5376, 65536]:
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert one(ctx, data) == (hashlib.md5(data).hexdigest(), zlib.crc32(data)), n


def test_quickpar_ifsc(ctx):
    qp = quickpar.load()
    src, owner = qp.slices()
    md5, crc = ctx.hash_slices([src[i] for i in range(len(src))], qp.block_size)
    for g, (fi, b) in enumerate(owner):
        want_md5, want_crc = qp.files[fi]["ifsc"][b]
        assert md5[g].tobytes().hex() == want_md5
        assert int(crc[g]) == want_crc


def test_many_slices_match_oracle(ctx):
    rng = np.random.default_rng(8)
    data = rng.integers(0, 256, (1000, 8192), dtype=np.uint8)
    md5, crc = ctx.hash_slices([data[i] for i in range(1000)], 8192)
    wmd5, wcrc = oracle.hash_slices(data)
    assert np.array_equal(md5, wmd5) and np.array_equal(crc, wcrc)


def test_slice_counts_and_chunk_edges(ctx):
    """Partial warps and CTAs (slices are hashed 32 to a warp, 256 to a CTA)
    and sizes on both sides of the 128-byte staging chunk and 64-byte block."""
    rng = np.random.default_rng(9)
    for n in (1, 31, 33, 257, 600):
        for S in (64, 127, 128, 129, 191, 192, 193, 255, 256, 384, 1000, 2050):
            data = rng.integers(0, 256, (n, S), dtype=np.uint8)
            md5, crc = ctx.hash_slices([data[i] for i in range(n)], S)
            wmd5, wcrc = oracle.hash_slices(data)
            assert np.array_equal(md5, wmd5) and np.array_equal(crc, wcrc), (n, S)


def test_verify_flags_damage(ctx):
    rng = np.random.default_rng(4)
    data = rng.integers(0, 256, (300, 4096), dtype=np.uint8)
    wmd5, wcrc = oracle.hash_slices(data)
    bad = data.copy()
    bad[[3, 50, 299]] = 0          # fully zeroed slices
    bad[7, 100] ^= 0x01            # single bit flip
    bad[120, 4095] ^= 0xFF
    ok = ctx.verify_slices([bad[i] for i in range(300)], 4096, wmd5, wcrc)
    assert set(np.flatnonzero(~ok).tolist()) == {3, 7, 50, 120, 299}


def test_device_pointers(ctx):
    import torch

    rng = np.random.default_rng(6)
    data = rng.integers(0, 256, (64, 65536), dtype=np.uint8)
    d = torch.from_numpy(data).cuda()
    md5, crc = ctx.hash_slices([d[i] for i in range(64)], 65536, device=True)
    wmd5, wcrc = oracle.hash_slices(data)
    assert np.array_equal(md5, wmd5) and np.array_equal(crc, wcrc)
