"""GPU parity of the repair path: device Gauss-Jordan (K2) and the two
multiply-accumulate passes, through the C ABI, against the oracle and the
QuickPar fixture (par2-rs tests/external_multiblock_repair.rs:50-247)."""
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


def par2_matrix(k, missing, exps):
    c = oracle.par2_constants(k)
    return np.array([[oracle.gf_pow(int(c[j]), int(e)) for j in missing] for e in exps], np.uint16)


def exponent_set(kind, m, rng):
    """run: 0..m-1 and offset/perm: a permuted run s..s+m-1 (closed-form
    Vandermonde inverse); gapped / gaps / far / below: a few exponents outside
    the best window (Woodbury correction above 96, Gauss-Jordan below)."""
    if kind == "run":
        return np.arange(m)
    if kind == "offset":
        return np.arange(7, 7 + m)
    if kind == "perm":
        return rng.permutation(np.arange(3, 3 + m))
    if kind == "gapped":
        return np.concatenate([np.arange(m - 1), [m + 4]])
    if kind == "gaps":       # lost recovery slices 2, 5, 9, 10 of the lowest m + 4
        keep = [e for e in range(m + 4) if e not in (2, 5, 9, 10)][:m]
        return rng.permutation(np.array(keep))
    if kind == "far":
        return np.array(([60000, 40001, 65534] + list(range(1, m)))[:m])
    return np.array(([0, 1] + list(range(50, 50 + m)))[:m])   # two below the window


@pytest.mark.parametrize("kind", ["run", "offset", "perm", "gapped", "gaps", "far", "below"])
@pytest.mark.parametrize("m", [1, 2, 13, 64, 96, 97, 130, 200, 333])
def test_reconstruction_matrix_matches_oracle(ctx, m, kind):
    rng = np.random.default_rng(m)
    k = 4 * m + 7
    missing = np.sort(rng.choice(k, m, replace=False))
    exps = exponent_set(kind, m, rng)
    got = ctx.reconstruction_matrix(k, missing, exps)
    want = oracle.invert(par2_matrix(k, missing, exps))
    assert want is not None
    assert np.array_equal(got, want)


def test_reconstruction_matrix_large_run(ctx):
    rng = np.random.default_rng(700)
    k, m = 3000, 700
    missing = np.sort(rng.choice(k, m, replace=False))
    exps = np.arange(m)
    assert np.array_equal(ctx.reconstruction_matrix(k, missing, exps),
                          oracle.invert(par2_matrix(k, missing, exps)))


@pytest.mark.parametrize("kind", ["run", "gapped", "woodbury"])
def test_repeated_constants_are_singular(ctx, kind):
    """Beyond 32768 slices the PAR2 constants repeat (c_i = c_{i+32768}):
    losing both slices of such a pair is unrepairable on either path."""
    import par2gpu

    k = 40000
    c = oracle.par2_constants(k)
    assert c[5] == c[5 + 32768]
    missing = np.array([5, 9, 5 + 32768])
    exps = np.arange(3) if kind == "run" else np.array([0, 1, 3])
    if kind == "woodbury":   # m = 150 with one exponent outside the window
        missing = np.sort(np.concatenate([[5, 5 + 32768], np.arange(100, 248)]))
        exps = np.concatenate([np.arange(149), [200]])
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.reconstruction_matrix(k, missing, exps)
    assert ei.value.code == par2gpu.ESINGULAR


def test_invert_random_and_singular(ctx):
    import par2gpu

    rng = np.random.default_rng(9)
    for m in (3, 17, 50):
        A = rng.integers(0, 65536, (m, m), dtype=np.uint16)
        want = oracle.invert(A)
        if want is None:
            continue
        assert np.array_equal(ctx.invert(A), want)
    # zero diagonal entries force the reference's row swap
    A = np.array([[0, 1, 2], [3, 0, 5], [7, 11, 0]], np.uint16)
    assert np.array_equal(ctx.invert(A), oracle.invert(A))
    S = np.array([[1, 2, 3], [2, 4, 6], [5, 6, 7]], np.uint16)
    S[1] = [oracle.gf_mul(2, int(v)) for v in S[0]]
    assert oracle.invert(S) is None
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.invert(S)
    assert ei.value.code == par2gpu.ESINGULAR
    assert "Singular matrix" in par2gpu.last_error()


def test_blocked_inversion_random_and_singular(ctx):
    """Matrices above the single-CTA size go through the blocked elimination
    (64-column panels whose row updates run on the multiply-accumulate
    kernel); singular ones must be reported, not faulted on."""
    import par2gpu

    rng = np.random.default_rng(12)
    for m in (100, 160, 257):
        A = rng.integers(0, 65536, (m, m), dtype=np.uint16)
        want = oracle.invert(A)
        assert want is not None
        assert np.array_equal(ctx.invert(A), want), m
    A = rng.integers(0, 65536, (150, 150), dtype=np.uint16)
    A[:, 70] = 0                       # a zero column in the second panel
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.invert(A)
    assert ei.value.code == par2gpu.ESINGULAR
    A = rng.integers(0, 65536, (200, 200), dtype=np.uint16)
    A[150] = A[3]                      # two equal rows
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.invert(A)
    assert ei.value.code == par2gpu.ESINGULAR
    # the context stays usable after a singular matrix
    B = rng.integers(0, 65536, (120, 120), dtype=np.uint16)
    assert np.array_equal(ctx.invert(B), oracle.invert(B))
    # invertible, but the leading 64 x 64 block of each panel's first unused
    # rows is singular (rows shuffled so that pivots sit far below): the panel
    # must fall back to searching for independent rows
    for m in (130, 200):
        A = rng.integers(0, 65536, (m, m), dtype=np.uint16)
        A[:64, :64] = 0
        A[64:128, 64:128] = 0 if m >= 128 else A[64:128, 64:128]
        A[5, :64] = A[7, :64]          # also a rank-deficient sub-block
        want = oracle.invert(A)
        assert want is not None
        assert np.array_equal(ctx.invert(A), want), m


def test_quickpar_repair_scenarios(ctx):
    qp = quickpar.load()
    src, _ = qp.slices()
    bs = qp.block_size
    t1 = qp.slice_base("test-1.data")
    t4 = qp.slice_base("test-4.data")
    n1 = (len(qp.files[qp.file_index("test-1.data")]["data"]) + bs - 1) // bs
    cases = {"single": [t1], "two_in_one": [t1, t1 + 3], "three_in_one": [t1, t1 + 2, t1 + 5],
             "two_files": [t1 + 1, t4 + 2], "deleted_file": list(range(t1, t1 + n1))}
    for name, dmg in cases.items():
        m = len(dmg)
        data = src.copy()
        data[dmg] = 0xAB
        rec = np.stack([qp.recovery[e] for e in range(m)])
        got = ctx.repair_array(data, dmg, np.arange(m), rec)
        assert np.array_equal(got, src[dmg]), name


@pytest.mark.parametrize("k,S,m", [(40, 4096, 1), (40, 4098, 5), (256, 8192, 13), (120, 6144, 60)])
def test_repair_matches_oracle(ctx, k, S, m):
    rng = np.random.default_rng(k + m)
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(m, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    missing = np.sort(rng.choice(k, m, replace=False))
    data = src.copy()
    data[missing] = 0
    want, moved = oracle.reconstruct(data, missing, exps, rec)
    got = ctx.repair_array(data, missing, exps, rec)
    assert np.array_equal(got, want)
    assert np.array_equal(got, src[missing])


@pytest.mark.parametrize("m", [7, 40])
def test_repair_from_host_buffers_in_upload_groups(ctx, m):
    """Host present slices (2048 - m of them, ragged 2050-byte slices) go up
    in 16 groups while the decode matrix forms and the earlier groups
    accumulate; the rebuilt slices equal the oracle's.  m = 7 runs the
    small-output records (24 words), m = 40 the 8 + 8 records (8 words), so
    both record strides pass through the per-group offsets."""
    rng = np.random.default_rng(77 + m)
    k, S = 2048, 2050
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(m, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    missing = np.sort(rng.choice(k, m, replace=False))
    data = src.copy()
    data[missing] = 0
    want, _ = oracle.reconstruct(data, missing, exps, rec)
    got = ctx.repair_array(data, missing, exps, rec)
    assert np.array_equal(got, want) and np.array_equal(got, src[missing])


@pytest.mark.parametrize("m", [13, 205])
def test_repair_from_host_buffers_with_slab_tail(ctx, m):
    """Wide host slices (1 MiB + 2 bytes): the last two upload groups run as
    column slabs -- each slab's present columns go up, both passes run on
    it, its rebuilt columns come back while the next slab uploads.  The
    rebuilt slices equal the erased ones (small-output and paired records)."""
    rng = np.random.default_rng(91 + m)
    k, S = 600, (1 << 20) + 2
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(m, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    missing = np.sort(rng.choice(k, m, replace=False))
    data = src.copy()
    data[missing] = 0
    got = ctx.repair_array(data, missing, exps, rec)
    assert np.array_equal(got, src[missing])


def test_singular_repair_while_uploads_are_in_flight(ctx):
    """Beyond 32768 slices the constants repeat, so losing slices 5 and
    5 + 32768 leaves a singular matrix: the host-buffer repair (present slices
    still going up in groups) reports it, and the context then repairs a
    normal set correctly."""
    import par2gpu

    k, S = 32780, 64
    data = np.zeros((k, S), np.uint8)
    rec = np.zeros((2, S), np.uint8)
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.repair_array(data, [5, 5 + 32768], np.arange(2, dtype=np.uint32), rec)
    assert ei.value.code == par2gpu.ESINGULAR and "Singular" in par2gpu.last_error()
    rng = np.random.default_rng(78)
    src = rng.integers(0, 256, (300, 4096), dtype=np.uint8)
    exps = np.arange(4, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    missing = [3, 150, 151, 299]
    broken = src.copy()
    broken[missing] = 0
    assert np.array_equal(ctx.repair_array(broken, missing, exps, rec), src[missing])


def test_repair_with_sparse_exponents(ctx):
    rng = np.random.default_rng(77)
    k, S = 64, 4096
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    all_exps = np.arange(20, dtype=np.uint32)
    rec = ctx.encode_array(src, all_exps)
    # recovery slices 0, 2, 3 were lost: the lowest surviving exponents are used
    avail = [e for e in range(20) if e not in (0, 2, 3)]
    missing = np.sort(rng.choice(k, 6, replace=False))
    use = np.array(avail[:6], np.uint32)
    data = src.copy()
    data[missing] = 0
    got = ctx.repair_array(data, missing, use, rec[use])
    want, _ = oracle.reconstruct(data, missing, use, rec[use])
    assert np.array_equal(got, want)
    assert np.array_equal(got, src[missing])


def test_plain_config_roundtrip(ctx):
    """16 MiB file, 64 KiB slices: k=256, r=13; zero 13 random slices and
    repair (the CPU-runnable plain configuration)."""
    rng = np.random.default_rng(2026)
    k, S, r = 256, 65536, 13
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    assert np.array_equal(rec, oracle.encode(src, exps))
    missing = np.sort(rng.choice(k, r, replace=False))
    data = src.copy()
    data[missing] = 0
    got = ctx.repair_array(data, missing, exps, rec)
    want, _ = oracle.reconstruct(data, missing, exps, rec)
    assert np.array_equal(got, want)
    assert np.array_equal(got, src[missing])


def test_repair_device_pointers(ctx):
    import torch

    rng = np.random.default_rng(5)
    k, S, m = 50, 8192, 7
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(m, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    missing = np.sort(rng.choice(k, m, replace=False))
    d_src = torch.from_numpy(src).cuda()
    d_rec = torch.from_numpy(rec).cuda()
    d_out = torch.zeros((m, S), dtype=torch.uint8, device="cuda")
    mset = set(missing.tolist())
    present = [d_src[i] for i in range(k) if i not in mset]
    ctx.repair(k, S, missing, present, exps, [d_rec[j] for j in range(m)],
               [d_out[j] for j in range(m)], device=True)
    assert np.array_equal(d_out.cpu().numpy(), src[missing])


def test_repair_argument_errors(ctx):
    import par2gpu

    data = np.zeros((4, 8), np.uint8)
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.repair(4, 8, [2, 1], [data[0], data[3]], [0, 1], [data[0], data[0]],
                   [data[1], data[2]])
    assert ei.value.code == par2gpu.EINVAL
