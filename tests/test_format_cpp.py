"""The PAR2 on-disk format (par2-rs_b200/host/par2_format.hpp, driven by
tests/cpp/test_format.cpp) against the QuickPar fixture set bundled with
par2-rs: the parser reads the set as par2-rs does (parser.rs:181-800), the
writer's packets are byte-identical to QuickPar's (every header holds the MD5
of its body), the files follow par2-rs's layout and names (creator.rs:453-521,
volumes.rs:65-210), and a created set repairs damaged files."""
import json
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from tests import quickpar

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "cpp", "_build", "test_format")
MAGIC = b"PAR2\x00PKT"
T_CREATOR = b"PAR 2.0\x00Creator\x00"
T_MAIN = b"PAR 2.0\x00Main\x00\x00\x00\x00"
T_DESC = b"PAR 2.0\x00FileDesc"
T_IFSC = b"PAR 2.0\x00IFSC\x00\x00\x00\x00"
T_RECV = b"PAR 2.0\x00RecvSlic"


def run(*args, check=True):
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpp")], check=True)
    p = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=600)
    if check:
        assert p.returncode == 0, p.stdout + p.stderr
    return p


def packet_headers(buf):
    """(type, header, exponent or None) of the packets of a file, in order."""
    out, pos = [], 0
    while pos + 64 <= len(buf):
        assert buf[pos:pos + 8] == MAGIC, pos
        (n,) = struct.unpack_from("<Q", buf, pos + 8)
        t = buf[pos + 48:pos + 64]
        e = struct.unpack_from("<I", buf, pos + 64)[0] if t == T_RECV else None
        out.append((t, buf[pos:pos + 64], e))
        pos += n
    assert pos == len(buf)
    return out


def test_calculate_block_size_matches_reference_tests():
    """creator.rs:539-585 (test_calculate_block_size): its known answers and
    its properties -- a multiple of 4, at least 2 KiB, at most 4 MiB up to
    260 GB of data, never more than 65535 slices -- for the C++ product's
    calculate_block_size (host only)."""
    sizes = [0, 1000, 1_000_000, 10_000_000, 100_000_000, 1_000_000_000, 10_000_000_000,
             260_000_000_000, 500_000_000_000, 2 ** 45 + 3]
    got = [int(x) for x in run("blocksize", *sizes).stdout.split()]
    bs = dict(zip(sizes, got))
    assert bs[0] == 2048 and bs[1_000_000] == 2048
    assert bs[10_000_000] == 5000 and bs[1_000_000_000] == 500_000
    for n, b in bs.items():
        assert b % 4 == 0 and b >= 2048, (n, b)
        if n <= 260_000_000_000:
            assert b <= 4 * 1024 * 1024, (n, b)
        if n:
            assert -(-n // b) <= 65535, (n, b)


def test_volume_rules_match_reference_tests():
    """volumes.rs:214-367: padding widths, volume file names, the Single and
    Exponential splits (1, 2, 4, ... slices per file), padding by the largest
    exponent, no volume for no recovery slices, the parent directory kept
    (host only)."""
    assert run("padwidth", 0, 9, 10, 99, 100, 999, 1000).stdout.split() == \
        ["1", "1", "2", "2", "3", "3", "4"]
    names = [("test", 0, 0, 1, "test.vol0+1.par2"), ("test", 0, 1, 1, "test.vol0+2.par2"),
             ("test", 0, 9, 2, "test.vol00+10.par2"), ("test", 10, 19, 2, "test.vol10+10.par2"),
             ("archive", 0, 99, 3, "archive.vol000+100.par2")]
    for base, a, b, w, want in names:
        assert run("volname", base, a, b, w).stdout.strip() == want

    def vols(scheme, n, base):
        out = run("volumes", scheme, n, base).stdout.splitlines()
        return [(int(a), int(b), int(c), p) for a, b, c, p in (line.split(" ", 3) for line in out)]

    v = vols("single", 3, "test")
    assert len(v) == 1 and v[0][:3] == (0, 2, 3) and v[0][3].endswith("vol0+3.par2")
    v = vols("exp", 7, "test")
    assert [x[:3] for x in v] == [(0, 0, 1), (1, 2, 2), (3, 6, 4)]
    assert [os.path.basename(x[3]) for x in v] == \
        ["test.vol0+1.par2", "test.vol1+2.par2", "test.vol3+4.par2"]
    for _, _, _, p in vols("exp", 100, "test"):
        assert len(os.path.basename(p)[len("test.vol"):].split("+")[0]) == 2, p
    assert vols("single", 0, "test") == []
    v = vols("single", 1, "/some/dir/test")
    assert len(v) == 1 and v[0][3].startswith("/some/dir/") and "test.vol" in v[0][3]


@pytest.fixture
def qp(tmp_path):
    q = quickpar.load()
    q.materialize(str(tmp_path))
    return q, tmp_path


def test_parse_quickpar_set(qp):
    q, d = qp
    p = json.loads(run("parse", d / "testdata.par2").stdout)
    assert p["block_size"] == q.block_size
    assert [f["name"] for f in p["files"]] == [f["name"] for f in q.files]  # Main order
    for f, g in zip(p["files"], q.files):
        assert (f["file_id"], f["length"], f["md5"], f["md5_16k"]) == \
            (g["file_id"], g["length"], g["md5"], g["md5_16k"])
        assert f["ifsc"] == g["ifsc"]
    # every volume's recovery slices, found by recovery set ID
    rec = dict(p["recovery"])
    assert sorted(rec) == list(range(60))
    assert all(rec[e] == q.recovery_md5[e] for e in rec)


def test_recovery_block_count_matches_reference():
    """creator.rs:323-327 (floor of data bytes x percent, then a ceiling
    division by the slice size): 57 % of 7 slices is 4 (tests/verify.rs
    test_missing_file_recreation_with_volumes), the plain and large
    configurations' 13 and 205, 0 % gives none, 100 % as many as data."""
    cases = [((7, 2048, 57), 4), ((256, 65536, 5), 13), ((2048, 1 << 20, 10), 205),
             ((40, 2048, 0), 0), ((22, 4096, 100), 22), ((53, 65536, 70), 38)]
    for (k, bs, pct), want in cases:
        assert run("reccount", k, bs, pct).stdout.strip() == str(want), (k, bs, pct)


def test_file_id_order_is_little_endian():
    """parser.rs:892-902: IDs compare from byte 15 down (par2cmdline's
    little-endian order), so a high last byte outranks a high first byte."""
    a = "ff" + "00" * 15
    b = "00" * 15 + "01"
    assert run("idless", a, b).stdout.strip() == "1"
    assert run("idless", b, a).stdout.strip() == "0"
    assert run("idless", a, a).stdout.strip() == "0"


def test_parse_from_a_volume_deduplicates_file_descriptions(qp):
    """parser.rs:921-954: a volume file repeats every FileDesc packet (vol31+29
    carries each of the 10 five times); loading the set from it yields one
    entry per file, in the Main packet's order, with all 60 recovery slices."""
    q, d = qp
    p = json.loads(run("parse", d / "testdata.vol31+29.par2").stdout)
    ids = [f["file_id"] for f in p["files"]]
    assert len(ids) == 10 and len(set(ids)) == 10
    assert [f["name"] for f in p["files"]] == [f["name"] for f in q.files]
    assert sorted(e for e, _ in p["recovery"]) == list(range(60))


def test_parser_skips_corrupt_packets_and_garbage(qp):
    q, d = qp
    buf = bytearray(open(d / "testdata.par2", "rb").read())
    hdrs = packet_headers(bytes(buf))
    # flip a byte inside the first IFSC body; insert garbage after the first packet
    off = 0
    for t, h, _ in hdrs:
        if t == T_IFSC:
            break
        off += struct.unpack_from("<Q", h, 8)[0]
    bad_id = bytes(buf[off + 64:off + 80]).hex()
    buf[off + 100] ^= 0xFF
    (n0,) = struct.unpack_from("<Q", hdrs[0][1], 8)
    buf[n0:n0] = b"PAR2\x00PK" + bytes(range(37))
    open(d / "testdata.par2", "wb").write(bytes(buf))
    p = json.loads(run("parse", d / "testdata.par2").stdout)
    assert [f["name"] for f in p["files"]] == [f["name"] for f in q.files]
    for f, g in zip(p["files"], q.files):
        assert f["ifsc"] == ([] if f["file_id"] == bad_id else g["ifsc"])


def test_main_and_file_desc_packets_match_quickpar(qp):
    q, d = qp
    got = [bytes.fromhex(x) for x in
           run("headers", d, q.block_size, *[f["name"] for f in q.files]).stdout.split()]
    fixture = {h for h, _ in q.packets}
    assert len(got) == 11 and all(h in fixture for h in got)


def test_missing_input_rejected(tmp_path):
    p = run("create", tmp_path / "x.par2", 0, 5, "exp", tmp_path / "missing.bin", check=False)
    assert p.returncode == 1 and "Input file does not exist" in p.stderr


@pytest.mark.gpu
def test_create_writes_quickpar_packets_in_par2_rs_layout(qp, tmp_path):
    """The QuickPar set recreated (same files, 5376-byte slices, 60 recovery
    slices): every packet but the Creator is byte-identical to QuickPar's,
    and the files are those par2-rs writes."""
    q, src = qp
    out = tmp_path / "out"
    out.mkdir()
    for f in q.files:
        shutil.copy(src / f["name"], out / f["name"])
    written = run("create", out / "testdata.par2", q.block_size, 30, "exp",
                  *[out / f["name"] for f in q.files]).stdout.split()
    names = sorted(os.path.basename(w) for w in written)
    assert names == sorted(f["name"] for f in q.par2_files)
    fixture = {h for h, _ in q.packets}
    want_exps = {"testdata.par2": []}
    for n in names[1:]:
        a, c = n[len("testdata.vol"):-len(".par2")].split("+")
        want_exps[n] = list(range(int(a), int(a) + int(c)))
    for w in written:
        hdrs = packet_headers(open(w, "rb").read())
        types = [t for t, _, _ in hdrs]
        nrec = len(want_exps[os.path.basename(w)])
        assert types == [T_CREATOR, T_MAIN] + [T_DESC] * 10 + [T_IFSC] * 10 + [T_RECV] * nrec
        assert [e for _, _, e in hdrs if e is not None] == want_exps[os.path.basename(w)]
        for t, h, _ in hdrs[1:]:
            assert h in fixture, (os.path.basename(w), t)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["single", "exp"])
def test_create_damage_repair_roundtrip(tmp_path, scheme):
    rng = np.random.default_rng(11)
    names = []
    for i, n in enumerate([0, 1, 4096, 10000, 65536, 123457, 300001]):
        name = f"file{i}.bin"
        (tmp_path / name).write_bytes(rng.integers(0, 256, n, dtype=np.uint8).tobytes())
        names.append(name)
    orig = {n: (tmp_path / n).read_bytes() for n in names}
    # 126 slices of 4096 bytes, 20 %: 26 recovery slices
    written = run("create", tmp_path / "set.par2", 4096, 20, scheme,
                  *[tmp_path / n for n in names]).stdout.split()
    assert os.path.basename(written[0]) == "set.par2"
    p = json.loads(run("parse", tmp_path / "set.par2").stdout)
    assert sorted(f["name"] for f in p["files"]) == sorted(names)
    assert p["block_size"] == 4096
    # lose one file, damage three slices of another
    os.unlink(tmp_path / "file4.bin")
    b = bytearray(orig["file6.bin"])
    for off in (5, 4096 * 20 + 7, len(b) - 1):
        b[off] ^= 0x5A
    (tmp_path / "file6.bin").write_bytes(bytes(b))
    r = run("repair", tmp_path / "set.par2", tmp_path).stdout.split("\n")
    assert r[0] == "damaged 19" and r[1] == "repaired 19"
    for n in names:
        assert (tmp_path / n).read_bytes() == orig[n], n
    assert run("repair", tmp_path / "set.par2", tmp_path).stdout.split("\n")[0] == "damaged 0"
