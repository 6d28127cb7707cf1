"""Pins the CPU oracle (oracle/par2_oracle.c) before anything is compared
against it:

* the GF(2^16) known answers of par2-rs tests/galois/core.rs and
  src/galois/tests.rs:7-89;
* the MD5/CRC32 known answers of src/hash/mod.rs:33-67;
* the QuickPar fixture set (tests/golden/quickpar.json): all 60 recovery
  slices (src/parser.rs:957-1021 checks exponents 0,1,2,3,5; here all 60),
  every IFSC entry, and the byte-exact repairs of
  tests/external_multiblock_repair.rs:50-247.
"""
import numpy as np
import pytest

from oracle import oracle as o
from tests import quickpar


def test_gf_known_answers():
    assert o.gf_mul(1, 5) == 5 and o.gf_mul(5, 1) == 5
    assert o.gf_mul(0, 5) == 0 and o.gf_mul(5, 0) == 0
    assert o.gf_mul(3, 7) == o.gf_mul(7, 3)
    assert o.gf_mul(123, 456) == o.gf_mul(456, 123)
    a, b, c = 1234, 5678, 9012
    assert o.gf_mul(o.gf_mul(a, b), c) == o.gf_mul(a, o.gf_mul(b, c))
    assert o.gf_div(5, 5) == 1 and o.gf_div(1234, 1234) == 1
    assert o.gf_div(5, 1) == 5 and o.gf_div(0, 5) == 0
    assert o.gf_div(o.gf_mul(a, b), b) == a
    assert o.gf_div(5, 0) is None and o.gf_div(0, 0) is None
    assert o.gf_pow(5, 0) == 1 and o.gf_pow(0, 0) == 1 and o.gf_pow(0, 100) == 0
    assert o.gf_pow(1234, 1) == 1234
    assert o.gf_pow(a, 2) == o.gf_mul(a, a)
    assert o.gf_pow(a, 7) == o.gf_mul(o.gf_pow(a, 3), o.gf_pow(a, 4))
    assert [o.gf_pow(2, n) for n in range(5)] == [1, 2, 4, 8, 16]
    for v in (2, 3, 1234, 65535):
        assert o.gf_mul(v, o.gf_pow(v, 65534)) == 1


def test_par2_constants():
    # par2_rs.rs:64-76: 2^n, n = 1, 2, 4, 7, 8, 11, ... (n coprime to 65535)
    assert list(o.par2_constants(6)) == [2, 4, 16, 128, 256, 2048]
    c = o.par2_constants(32768)
    assert len(set(c.tolist())) == 32768  # all distinct within the field's limit


def test_hash_known_answers():
    assert o.md5(b"").hex() == "d41d8cd98f00b204e9800998ecf8427e"
    assert o.md5(b"abc").hex() == "900150983cd24fb0d6963f7d28e17f72"
    assert o.md5(b"message digest").hex() == "f96b697d7cb7938d525a2f31aaf161d0"
    assert o.crc32(b"") == 0
    assert o.crc32(b"abc") == 0x352441C2


@pytest.fixture(scope="module")
def qp():
    return quickpar.load()


def test_quickpar_all_recovery_slices(qp):
    src, _ = qp.slices()
    assert src.shape == (200, 5376)
    exps = np.arange(60, dtype=np.uint32)
    rec = o.encode(src, exps)
    for e in range(60):
        assert np.array_equal(rec[e], qp.recovery[e]), f"exponent {e}"


def test_quickpar_ifsc(qp):
    src, owner = qp.slices()
    md5s, crcs = o.hash_slices(src)
    for g, (fi, b) in enumerate(owner):
        want_md5, want_crc = qp.files[fi]["ifsc"][b]
        assert md5s[g].tobytes().hex() == want_md5
        assert int(crcs[g]) == want_crc


def _repair_case(qp, damaged_global):
    """Repair `damaged_global` slices with the lowest-exponent recovery slices
    (repair.rs:585-604) and return (rebuilt, pristine)."""
    src, _ = qp.slices()
    missing = sorted(damaged_global)
    m = len(missing)
    exps = np.arange(m, dtype=np.uint32)
    rec = np.stack([qp.recovery[e] for e in range(m)])
    data = src.copy()
    data[missing] = 0xAB  # damaged contents must not matter
    out, moved = o.reconstruct(data, missing, exps, rec, ref_row_quirk=True)
    return out, src[missing], moved


def test_quickpar_repair_scenarios(qp):
    bs = qp.block_size
    t1 = qp.slice_base("test-1.data")
    t4 = qp.slice_base("test-4.data")
    cases = {
        "single": [t1 + 0],
        "two_in_one": [t1 + 0, t1 + 3],
        "three_in_one": [t1 + 0, t1 + 2, t1 + 5],
        "two_files": [t1 + 1, t4 + 2],
        "deleted_file": list(range(t1, t1 + (len(qp.files[qp.file_index("test-1.data")]["data"]) + bs - 1) // bs)),
    }
    for name, dmg in cases.items():
        out, pristine, moved = _repair_case(qp, dmg)
        assert out is not None, name
        assert moved == 0, name
        assert np.array_equal(out, pristine), name


def test_invert_roundtrip():
    rng = np.random.default_rng(3)
    c = o.par2_constants(40)
    for m in (1, 2, 5, 13):
        cols = rng.choice(40, m, replace=False)
        A = np.array([[o.gf_pow(int(c[j]), e) for j in cols] for e in range(m)], np.uint16)
        Ainv = o.invert(A)
        assert Ainv is not None
        # A * Ainv == I over GF(2^16)
        for i in range(m):
            for j in range(m):
                acc = 0
                for t in range(m):
                    acc ^= o.gf_mul(int(A[i, t]), int(Ainv[t, j]))
                assert acc == (1 if i == j else 0)


def test_singular_matrix_detected():
    A = np.array([[1, 2], [1, 2]], np.uint16)
    assert o.invert(A) is None
    # duplicate missing column -> singular repair ("Singular matrix",
    # par2_rs.rs:361-370)
    data = np.zeros((4, 8), np.uint8)
    out, _ = o.reconstruct(data, [1, 1], [0, 1], np.zeros((2, 8), np.uint8))
    assert out is None


def test_creator_rules():
    # creator.rs:540-585 style checks of the block-size rule
    assert o.calculate_block_size(0) == 2048
    assert o.calculate_block_size(1000) == 2048
    # creator.rs:541-544
    assert o.calculate_block_size(1_000_000) == 2048
    assert o.calculate_block_size(10_000_000) == 5000
    assert o.calculate_block_size(1_000_000_000) == 500_000
    assert o.calculate_block_size(2000 * 8192) == 8192
    assert o.calculate_block_size(10 ** 12) % 4 == 0
    bs = o.calculate_block_size(10 ** 13)
    assert (10 ** 13 + bs - 1) // bs <= 65535
    # 16 MiB at 64 KiB and 5 % -> 13 recovery slices; 2 GiB at 1 MiB, 10 % -> 205
    assert o.recovery_count(256, 65536, 5.0) == 13
    assert o.recovery_count(2048, 1 << 20, 10.0) == 205
    assert o.recovery_count(32000, 65536, 5.0) == 1600


def test_cpu_baseline_matches_oracle():
    rng = np.random.default_rng(7)
    src = rng.integers(0, 256, (37, 4096 + 34), dtype=np.uint8)
    want = o.encode(src, np.arange(11, dtype=np.uint32))
    got = o.cpu_encode(src, 11, 4)
    assert np.array_equal(want, got)
