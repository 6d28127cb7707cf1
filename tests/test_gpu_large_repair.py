"""GPU parity at the high-slice-count verify + repair size: 32000 source
slices, 1600 erasures (par2_rs.rs:319-422 transform, :442-675 reconstruction,
verify.rs:548-654 per-slice checks).

* The 1600 x 1600 decode matrix from each device path (closed-form
  Vandermonde inverse, its Woodbury correction, the blocked Gauss-Jordan of
  p2g_invert) equals the oracle's elimination of the same matrix entry for
  entry, and A x (A^-1 v) = v holds for random vectors v (checked on the
  host in numpy; a wrong inverse passes one vector with probability
  1/65536).
* A 32000 x 4 KiB set with 1600 recovery slices: the recovery slices equal
  the restated par2-rs AVX2 strategy's (itself checked against the oracle on
  the CPU), the device verify finds exactly the 1600 damaged slices (800
  zeroed, 800 with 1-64 flipped bytes), and the repair rebuilds every one of
  them byte for byte.  The reference's own repair output is the pristine data
  whenever the matrix is invertible, so the pristine slices are the oracle's
  answer at this size, where the scalar oracle would take hours.
"""
import hashlib
import os
import zlib

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

K, M = 32000, 1600


@pytest.fixture(scope="module")
def ctx():
    import par2gpu

    c = par2gpu.Context(0)
    yield c
    c.close()


def _gf_tables():
    exp = oracle.power_matrix(np.array([2], np.uint16), np.arange(65535, dtype=np.uint32))[:, 0]
    log = np.zeros(65536, np.int64)
    log[exp] = np.arange(65535)
    return exp.astype(np.int64), log


def _gf_matvec(A, v, exp, log):
    """A (n x n) times v over GF(2^16), row by row in numpy."""
    out = np.zeros(A.shape[0], np.int64)
    nz = v != 0
    lv = log[v[nz]]
    for r in range(A.shape[0]):
        a = A[r, nz].astype(np.int64)
        keep = a != 0
        prods = exp[(log[a[keep]] + lv[keep]) % 65535]
        out[r] = np.bitwise_xor.reduce(prods) if len(prods) else 0
    return out


def _check_inverse(A, Ainv, rng, nvec=2):
    exp, log = _gf_tables()
    for _ in range(nvec):
        v = rng.integers(0, 65536, A.shape[0]).astype(np.int64)
        assert np.array_equal(_gf_matvec(A, _gf_matvec(Ainv, v, exp, log), exp, log), v)


@pytest.mark.parametrize("kind", ["consecutive", "one_off", "general"])
def test_decode_matrix_m1600_matches_oracle(ctx, kind):
    rng = np.random.default_rng({"consecutive": 1, "one_off": 2, "general": 3}[kind])
    missing = np.sort(rng.choice(K, M, replace=False))
    if kind == "consecutive":     # the m lowest exponents of an undamaged set
        exps = np.arange(M)
    elif kind == "one_off":       # recovery slice 17 lost: the next one stands in
        exps = np.concatenate([np.arange(17), np.arange(18, M + 1)])
    else:                         # 200 exponents far outside any window: elimination
        exps = np.concatenate([np.arange(M - 200), 30000 + 7 * np.arange(200)])
    A = oracle.erasure_matrix(K, missing, exps)
    if kind == "general":
        got = ctx.invert(A)
    else:
        got = ctx.reconstruction_matrix(K, missing, exps)
    want = oracle.invert(A)
    assert want is not None
    assert np.array_equal(got, want)
    _check_inverse(A, got, rng)


def test_repair_1600_of_32000_slices(ctx):
    import torch

    S = 4096
    rng = np.random.default_rng(32000)
    src_np = rng.integers(0, 256, (K, S), dtype=np.uint8)
    dev = torch.device("cuda", 0)
    src = torch.from_numpy(src_np).to(dev)
    rec = torch.zeros((M, S), dtype=torch.uint8, device=dev)
    exps = np.arange(M, dtype=np.uint32)
    ctx.encode(src, S, exps, rec, device=True)
    torch.cuda.synchronize()
    want_rec = oracle.cpu_encode(src_np, M, os.cpu_count() or 1)
    assert np.array_equal(rec.cpu().numpy(), want_rec)

    # IFSC checksums of the pristine slices from the device, checked on a sample
    md5, crc = ctx.hash_slices(src, S, device=True)
    for i in rng.choice(K, 64, replace=False):
        assert bytes(md5[i]) == hashlib.md5(src_np[i].tobytes()).digest()
        assert int(crc[i]) == zlib.crc32(src_np[i].tobytes())

    # damage: 800 slices zeroed, 800 with 1-64 flipped bytes
    dmg = np.sort(rng.choice(K, M, replace=False))
    damaged = src_np.copy()
    damaged[dmg[: M // 2]] = 0
    for i in dmg[M // 2:]:
        n = int(rng.integers(1, 65))
        offs = rng.choice(S, n, replace=False)
        damaged[i, offs] ^= rng.integers(1, 256, n, dtype=np.uint8)
    assert not np.array_equal(damaged[dmg[M // 2]], src_np[dmg[M // 2]])
    src.copy_(torch.from_numpy(damaged))
    ok = ctx.verify_slices(src, S, md5, crc, device=True)
    assert np.array_equal(np.flatnonzero(~ok), dmg)

    keep = np.ones(K, bool)
    keep[dmg] = False
    present = np.uint64(src.data_ptr()) + np.flatnonzero(keep).astype(np.uint64) * np.uint64(S)
    fixed = torch.zeros((M, S), dtype=torch.uint8, device=dev)
    ctx.repair(K, S, dmg, present, exps, rec, fixed, device=True)
    torch.cuda.synchronize()
    assert np.array_equal(fixed.cpu().numpy(), src_np[dmg])
