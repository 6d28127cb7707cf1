"""The create / repair pipelines through their C ABI (include/par2format.h,
libpar2format.so): Par2Creator::create and Par2Repairer::repair of par2-rs
over files, with the slices streamed into device memory."""
import os

import numpy as np
import pytest

from par2gpu import format as fmt


def make_files(d, sizes, seed):
    rng = np.random.default_rng(seed)
    names = []
    for i, n in enumerate(sizes):
        p = d / f"part{i}.bin"
        p.write_bytes(rng.integers(0, 256, n, dtype=np.uint8).tobytes())
        names.append(p)
    return names


def test_errors_without_work(tmp_path):
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.create([tmp_path / "missing.bin"])
    assert ei.value.code == fmt.ERROR and "Input file does not exist" in str(ei.value)
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.create([])
    assert "No input files" in str(ei.value)
    (tmp_path / "a.bin").write_bytes(b"x" * 10)
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.create([tmp_path / "a.bin"], block_size=2050)
    assert "multiple of 4" in str(ei.value)
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair(tmp_path / "none.par2", tmp_path)
    assert ei.value.code == fmt.ERROR


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [fmt.SCHEME_SINGLE, fmt.SCHEME_EXPONENTIAL])
def test_create_damage_repair(tmp_path, scheme):
    sizes = [0, 3, 100000, 1 << 20, (1 << 20) + 17, 5 * 65536, 777777]
    files = make_files(tmp_path, sizes, 21)
    orig = {p.name: p.read_bytes() for p in files}
    # 53 slices of 64 KiB, 70 %: 38 recovery slices for the 32 damaged below
    st = fmt.create(files, tmp_path / "set.par2", block_size=65536, redundancy=70, scheme=scheme)
    assert st.bytes_read == sum(sizes) and st.block_size == 65536
    assert st.data_blocks == sum((n + 65535) // 65536 for n in sizes)
    assert st.recovery_blocks == (int(st.data_blocks * 65536 * 0.7) + 65535) // 65536 == 38
    assert (tmp_path / "set.par2").exists()
    n, st = fmt.repair(tmp_path / "set.par2", tmp_path)
    assert n == 0 and st.damaged_blocks == 0
    # a lost file, a truncated file and flipped bytes in a third
    os.unlink(tmp_path / "part3.bin")
    (tmp_path / "part4.bin").write_bytes(orig["part4.bin"][:200000])
    b = bytearray(orig["part6.bin"])
    b[12345] ^= 1
    b[-1] ^= 0x80
    (tmp_path / "part6.bin").write_bytes(bytes(b))
    n, st = fmt.repair(tmp_path / "set.par2", tmp_path)
    assert n == 16 + 14 + 2 and st.files_written == 3
    for p in files:
        assert p.read_bytes() == orig[p.name], p.name


@pytest.mark.gpu
def test_slices_and_files_larger_than_the_copy_chunks(tmp_path):
    """12 MiB slices and files of several 8 MiB copy chunks: the recovery
    slices are read and uploaded in pieces (two per slice), the recovery
    buffer and the rebuilt files come back in several chunks written at their
    offsets; the rebuilt bytes equal the originals."""
    sizes = [30 * (1 << 20) + 4321, 25 * (1 << 20)]
    files = make_files(tmp_path, sizes, 23)
    orig = {p.name: p.read_bytes() for p in files}
    bs = 12 << 20
    st = fmt.create(files, tmp_path / "big.par2", block_size=bs, redundancy=50)
    assert st.data_blocks == 3 + 3 and st.recovery_blocks == 3
    # a slice in the middle of the first file, the last (ragged) one, and
    # the second file's first slice
    b = bytearray(orig["part0.bin"])
    b[bs + 99] ^= 0xFF
    b[-1] ^= 1
    (tmp_path / "part0.bin").write_bytes(bytes(b))
    c = bytearray(orig["part1.bin"])
    c[7] ^= 0x10
    (tmp_path / "part1.bin").write_bytes(bytes(c))
    n, st = fmt.repair(tmp_path / "big.par2", tmp_path)
    assert n == 3 and st.files_written == 2
    for p in files:
        assert p.read_bytes() == orig[p.name], p.name


@pytest.mark.gpu
def test_insufficient_recovery(tmp_path):
    files = make_files(tmp_path, [1 << 20, 1 << 20], 22)
    fmt.create(files, tmp_path / "s.par2", block_size=65536, redundancy=5)  # 2 slices
    os.unlink(files[0])
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair(tmp_path / "s.par2", tmp_path)
    assert ei.value.code == fmt.EINSUFFICIENT


def test_cancel_before_start(tmp_path):
    import ctypes

    flag = ctypes.c_int32(1)
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "none.par2", tmp_path, cancel=flag)
    assert ei.value.code == fmt.ECANCELLED and "cancelled" in str(ei.value)


def _damaged_set(tmp_path, seed):
    files = make_files(tmp_path, [300000, 1 << 20, 123457], seed)
    orig = {p.name: p.read_bytes() for p in files}
    fmt.create(files, tmp_path / "set.par2", block_size=65536, redundancy=50,
               scheme=fmt.SCHEME_EXPONENTIAL)
    b = bytearray(orig["part1.bin"])
    b[70000] ^= 0xFF
    (tmp_path / "part1.bin").write_bytes(bytes(b))
    os.unlink(tmp_path / "part2.bin")
    return files, orig


@pytest.mark.gpu
def test_repair_ex_verify_only_progress_and_purge(tmp_path):
    files, orig = _damaged_set(tmp_path, 31)
    seen = []
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "set.par2", tmp_path, do_repair=False,
                      progress=lambda op, c, t: seen.append((op, c, t)))
    assert ei.value.code == fmt.EDAMAGED
    assert "repair was not requested" in str(ei.value)
    assert (fmt.OP_LOADING, 0, 100) in seen and (fmt.OP_VERIFYING, 100, 100) in seen
    assert (tmp_path / "part1.bin").read_bytes() != orig["part1.bin"]   # untouched
    seen.clear()
    par2s = sorted(p.name for p in tmp_path.iterdir() if p.suffix == ".par2")
    assert len(par2s) > 1
    n, st = fmt.repair_ex(tmp_path / "set.par2", tmp_path, purge=True,
                          progress=lambda op, c, t: seen.append((op, c, t)))
    assert n == 1 + 2 and st.files_written == 2
    assert (fmt.OP_REPAIRING, 100, 100) in seen
    for p in files:
        assert p.read_bytes() == orig[p.name]
    assert not [p for p in tmp_path.iterdir() if p.suffix in (".par2", ".par2tmp")]


@pytest.mark.gpu
def test_cancel_during_repair_leaves_files_unchanged(tmp_path):
    import ctypes

    files, orig = _damaged_set(tmp_path, 32)
    before = {p.name: p.read_bytes() for p in tmp_path.iterdir() if p.suffix == ".bin"}
    flag = ctypes.c_int32(0)

    def progress(op, cur, tot):
        if op == fmt.OP_REPAIRING and cur == 0:
            flag.value = 1

    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "set.par2", tmp_path, progress=progress, cancel=flag)
    assert ei.value.code == fmt.ECANCELLED
    after = {p.name: p.read_bytes() for p in tmp_path.iterdir() if p.suffix == ".bin"}
    assert after == before                       # nothing committed, nothing half-written
    assert not [p for p in tmp_path.iterdir() if p.suffix == ".par2tmp"]


@pytest.mark.gpu
def test_cancel_after_commit_skips_purge(tmp_path):
    import ctypes

    files, orig = _damaged_set(tmp_path, 33)
    flag = ctypes.c_int32(0)

    def progress(op, cur, tot):
        if op == fmt.OP_REPAIRING and cur == 100:
            flag.value = 1

    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "set.par2", tmp_path, purge=True, progress=progress, cancel=flag)
    assert ei.value.code == fmt.ECANCELLED
    for p in files:                               # the repair was committed
        assert p.read_bytes() == orig[p.name]
    assert (tmp_path / "set.par2").exists()       # but the purge was skipped


# ---- the reference's edge-case, error-path and robustness tests
# (tests/edge_cases.rs, tests/error_paths.rs, tests/robustness.rs) -------------

def test_block_size_below_minimum_rejected(tmp_path):
    """edge_cases.rs test_block_size_too_small: below 2 KiB is an error (0
    through this C ABI means "choose automatically")."""
    (tmp_path / "data.bin").write_bytes(b"DATA" * 2500)
    for bs in (4, 2044):
        with pytest.raises(fmt.Par2FormatError) as ei:
            fmt.create([tmp_path / "data.bin"], block_size=bs)
        assert "at least 2048" in str(ei.value)


@pytest.mark.parametrize("content", [b"", b"PAR2\x00PKT", b"\x00" * 4096])
def test_empty_truncated_and_garbage_par2_files(tmp_path, content):
    """error_paths.rs test_empty_par2_file / test_truncated_par2_file and
    edge_cases.rs test_invalid_par2_file: no set is read from them."""
    p = tmp_path / "bad.par2"
    p.write_bytes(content)
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair(p, tmp_path)
    assert ei.value.code == fmt.ERROR


@pytest.mark.gpu
def test_zero_redundancy(tmp_path):
    """edge_cases.rs test_zero_redundancy: a set with no recovery slices
    verifies intact files and cannot repair damage."""
    files = make_files(tmp_path, [5000 * 4], 24)
    st = fmt.create(files, tmp_path / "z.par2", redundancy=0)
    assert st.recovery_blocks == 0 and (tmp_path / "z.par2").exists()
    n, st = fmt.repair(tmp_path / "z.par2", tmp_path)
    assert n == 0 and st.damaged_blocks == 0
    b = bytearray(files[0].read_bytes())
    b[100:200] = b"\xff" * 100
    files[0].write_bytes(bytes(b))
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "z.par2", tmp_path, do_repair=False)
    assert ei.value.code == fmt.EDAMAGED
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair(tmp_path / "z.par2", tmp_path)
    assert ei.value.code == fmt.EINSUFFICIENT


@pytest.mark.gpu
@pytest.mark.parametrize("change", ["truncate", "extend"])
def test_truncated_and_extended_files(tmp_path, change):
    """edge_cases.rs test_truncated_file_detection / test_extended_file_
    detection: verification reports the file damaged; repair restores its
    exact length and bytes."""
    files = make_files(tmp_path, [10000 * 8], 25)
    orig = files[0].read_bytes()
    # 40 slices of 2 KiB, 24 recovery slices: the cut at 40000 bytes loses 21
    fmt.create(files, tmp_path / "t.par2", redundancy=60)
    files[0].write_bytes(orig[:40000] if change == "truncate" else orig + b"EXTRA_DATA")
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "t.par2", tmp_path, do_repair=False)
    assert ei.value.code == fmt.EDAMAGED
    n, st = fmt.repair(tmp_path / "t.par2", tmp_path)
    assert n >= 1
    assert files[0].read_bytes() == orig


@pytest.mark.gpu
def test_all_files_missing(tmp_path):
    """edge_cases.rs test_all_files_missing: with as many recovery slices as
    data slices, every file is recreated from the recovery slices alone."""
    files = make_files(tmp_path, [9000, 70000, 3], 26)
    orig = {p.name: p.read_bytes() for p in files}
    st = fmt.create(files, tmp_path / "all.par2", block_size=4096, redundancy=100)
    assert st.recovery_blocks >= st.data_blocks
    for p in files:
        os.unlink(p)
    n, st = fmt.repair(tmp_path / "all.par2", tmp_path)
    assert n == st.data_blocks and st.files_written == 3
    for p in files:
        assert p.read_bytes() == orig[p.name]


@pytest.mark.gpu
def test_many_small_files_and_monotonic_progress(tmp_path):
    """robustness.rs test_many_small_files_50, test_progress_never_exceeds_
    total and test_progress_monotonic_per_operation: 50 small files of mixed
    sizes, a few damaged; progress stays within its total and never goes
    back within an operation."""
    rng = np.random.default_rng(27)
    files = make_files(tmp_path, [int(x) for x in rng.integers(0, 20000, 50)], 27)
    orig = {p.name: p.read_bytes() for p in files}
    fmt.create(files, tmp_path / "many.par2", block_size=2048, redundancy=20)
    for i in (3, 17, 41):
        if orig[files[i].name]:
            b = bytearray(orig[files[i].name])
            b[len(b) // 2] ^= 0xA5
            files[i].write_bytes(bytes(b))
    seen = []
    n, st = fmt.repair_ex(tmp_path / "many.par2", tmp_path,
                          progress=lambda op, c, t: seen.append((op, c, t)))
    for p in files:
        assert p.read_bytes() == orig[p.name], p.name
    last = {}
    for op, c, t in seen:
        assert 0 <= c <= t, (op, c, t)
        assert c >= last.get(op, 0), (op, c, last)
        last[op] = c


def _strip_ifsc(directory, only_file_id=None):
    """Drops the IFSC packets (all, or those of one File ID) from every .par2
    file of a set, as a set made without slice checksums would be."""
    import struct

    for p in directory.iterdir():
        if p.suffix != ".par2":
            continue
        buf, out, pos = p.read_bytes(), bytearray(), 0
        while pos + 64 <= len(buf):
            (n,) = struct.unpack_from("<Q", buf, pos + 8)
            pkt = buf[pos:pos + n]
            is_ifsc = pkt[48:64] == b"PAR 2.0\x00IFSC\x00\x00\x00\x00"
            if not (is_ifsc and (only_file_id is None or pkt[64:80] == only_file_id)):
                out += pkt
            pos += n
        p.write_bytes(bytes(out))


def _file_ids(par2_path):
    """File ID of every FileDesc packet, by file name."""
    import struct

    buf, pos, ids = par2_path.read_bytes(), 0, {}
    while pos + 64 <= len(buf):
        (n,) = struct.unpack_from("<Q", buf, pos + 8)
        if buf[pos + 48:pos + 64] == b"PAR 2.0\x00FileDesc":
            body = buf[pos + 64:pos + n]
            ids[body[56:].split(b"\x00")[0].decode()] = body[:16]
        pos += n
    return ids


@pytest.mark.gpu
def test_sets_without_ifsc_fall_back_to_whole_file_md5(tmp_path):
    """verify.rs test_verification_without_ifsc(_detects_damage): with no IFSC
    packets an intact set verifies by the files' MD5s, and a damaged file is
    detected and rebuilt as a whole (no slice-level information)."""
    files = make_files(tmp_path, [10 * 2048 - 7, 40 * 2048], 28)
    orig = {p.name: p.read_bytes() for p in files}
    fmt.create(files, tmp_path / "n.par2", block_size=2048, redundancy=30)  # 15 slices
    _strip_ifsc(tmp_path)
    n, st = fmt.repair_ex(tmp_path / "n.par2", tmp_path, do_repair=False)
    assert n == 0 and st.damaged_blocks == 0
    b = bytearray(orig["part0.bin"])
    b[5000] ^= 0x01
    files[0].write_bytes(bytes(b))
    with pytest.raises(fmt.Par2FormatError) as ei:
        fmt.repair_ex(tmp_path / "n.par2", tmp_path, do_repair=False)
    assert ei.value.code == fmt.EDAMAGED
    n, st = fmt.repair(tmp_path / "n.par2", tmp_path)
    assert n == 10 and st.files_written == 1          # the whole damaged file
    for p in files:
        assert p.read_bytes() == orig[p.name], p.name


@pytest.mark.gpu
def test_mixed_ifsc_and_whole_file_verification(tmp_path):
    """One file without IFSC (checked by MD5), one with it (checked per
    slice): a single damaged slice of the second is the only one rebuilt."""
    files = make_files(tmp_path, [6 * 2048, 30 * 2048 + 99], 29)
    orig = {p.name: p.read_bytes() for p in files}
    fmt.create(files, tmp_path / "m.par2", block_size=2048, redundancy=20)
    _strip_ifsc(tmp_path, only_file_id=_file_ids(tmp_path / "m.par2")["part0.bin"])
    b = bytearray(orig["part1.bin"])
    b[2048 * 7 + 3] ^= 0x40
    files[1].write_bytes(bytes(b))
    n, st = fmt.repair(tmp_path / "m.par2", tmp_path)
    assert n == 1 and st.files_written == 1
    for p in files:
        assert p.read_bytes() == orig[p.name], p.name


# ---- cancellation on the QuickPar set (tests/info_and_cancel.rs:216-380) ------

def _qp_set(tmp_path):
    from tests import quickpar

    q = quickpar.load()
    q.materialize(str(tmp_path))
    return tmp_path / "testdata.par2"


def _data_files(d):
    return {p.name: p.read_bytes() for p in sorted(d.iterdir()) if p.suffix == ".data"}


def _corrupt(d, name, off, n, byte):
    b = bytearray((d / name).read_bytes())
    b[off:off + n] = bytes([byte]) * n
    (d / name).write_bytes(bytes(b))


@pytest.mark.gpu
def test_preset_cancel_leaves_damaged_files_unchanged(tmp_path):
    """test_repair_cancellation_preset_flag_is_safe and
    test_verify_cancellation_preset_flag."""
    import ctypes

    index = _qp_set(tmp_path)
    for name in ("test-1.data", "test-6.data"):
        _corrupt(tmp_path, name, 2048, 8192, 0xAB)
    before = _data_files(tmp_path)
    for do_repair in (True, False):
        with pytest.raises(fmt.Par2FormatError) as ei:
            fmt.repair_ex(index, tmp_path, do_repair=do_repair, purge=True,
                          cancel=ctypes.c_int32(1))
        assert ei.value.code == fmt.ECANCELLED
        assert _data_files(tmp_path) == before
    assert index.exists()


@pytest.mark.gpu
@pytest.mark.parametrize("delay_us", [0, 50, 500, 5000])
def test_cancel_from_another_thread(tmp_path, delay_us):
    """test_repair_cancellation_from_thread_is_safe: whichever stage the flag
    lands in, the call either reports ECANCELLED with the data files
    untouched, or completes with the file repaired and no temp file left."""
    import ctypes
    import threading
    import time

    index = _qp_set(tmp_path)
    orig = _data_files(tmp_path)
    _corrupt(tmp_path, "test-4.data", 512, 16384, 0xCD)
    before = _data_files(tmp_path)
    flag = ctypes.c_int32(0)

    def setter():
        time.sleep(delay_us * 1e-6)
        flag.value = 1

    t = threading.Thread(target=setter)
    t.start()
    try:
        fmt.repair_ex(index, tmp_path, cancel=flag)
        assert _data_files(tmp_path) == orig
    except fmt.Par2FormatError as e:
        assert e.code == fmt.ECANCELLED, e
        assert _data_files(tmp_path) in (before, orig)   # untouched, or committed
    finally:
        t.join()
    assert not [p for p in tmp_path.iterdir() if p.suffix == ".par2tmp"]


@pytest.mark.gpu
def test_unset_cancel_flag_repairs_normally(tmp_path):
    """test_normal_cancellable_repair_succeeds_with_flag_unset."""
    import ctypes

    index = _qp_set(tmp_path)
    orig = _data_files(tmp_path)
    _corrupt(tmp_path, "test-2.data", 100, 1000, 0x00)
    n, st = fmt.repair_ex(index, tmp_path, cancel=ctypes.c_int32(0))
    assert n == 1 and _data_files(tmp_path) == orig


# ---- progress (tests/progress.rs) ---------------------------------------------

@pytest.mark.gpu
def test_progress_operations_of_repair_and_verify(tmp_path):
    """test_progress_callbacks_during_repair / _verify_only: repair reports
    Scanning, Loading, Verifying and Repairing with a non-zero total and
    current <= total; verify-only never reports Repairing."""
    files = make_files(tmp_path, [50000 * 4], 30)
    fmt.create(files, tmp_path / "p.par2", redundancy=20)
    b = bytearray(files[0].read_bytes())
    b[1000:6000] = b"\xff" * 5000
    files[0].write_bytes(bytes(b))
    seen = []
    fmt.repair_ex(tmp_path / "p.par2", tmp_path, progress=lambda *a: seen.append(a))
    ops = {op for op, _, _ in seen}
    assert ops >= {fmt.OP_SCANNING, fmt.OP_LOADING, fmt.OP_VERIFYING, fmt.OP_REPAIRING}
    assert all(t > 0 and c <= t for _, c, t in seen)
    seen.clear()
    fmt.repair_ex(tmp_path / "p.par2", tmp_path, do_repair=False, progress=lambda *a: seen.append(a))
    ops = {op for op, _, _ in seen}
    assert ops >= {fmt.OP_SCANNING, fmt.OP_LOADING, fmt.OP_VERIFYING}
    assert fmt.OP_REPAIRING not in ops


@pytest.mark.gpu
def test_verify_only_with_purge_removes_the_set(tmp_path):
    """test_progress_callbacks_with_purge: a verify-only run over intact
    files with purge set removes every .par2 file of the set."""
    files = make_files(tmp_path, [20000], 31)
    fmt.create(files, tmp_path / "q.par2", redundancy=10)
    assert [p for p in tmp_path.iterdir() if p.suffix == ".par2"]
    seen = []
    n, st = fmt.repair_ex(tmp_path / "q.par2", tmp_path, do_repair=False, purge=True,
                          progress=lambda *a: seen.append(a))
    assert n == 0 and fmt.OP_VERIFYING in {op for op, _, _ in seen}
    assert not [p for p in tmp_path.iterdir() if p.suffix == ".par2"]


@pytest.mark.gpu
def test_creator_progress_reaches_the_total(tmp_path):
    """robustness.rs test_creator_progress_callbacks: creation reports
    encoding progress (as Repairing, the reference's name for it) from 0 to
    the number of data slices."""
    files = make_files(tmp_path, [200000], 32)
    seen = []
    st = fmt.create(files, tmp_path / "c.par2", redundancy=10,
                    progress=lambda *a: seen.append(a))
    enc = [(c, t) for op, c, t in seen if op == fmt.OP_REPAIRING]
    assert enc and enc[0] == (0, st.data_blocks) and enc[-1] == (st.data_blocks, st.data_blocks)
    assert all(a[0] <= b[0] for a, b in zip(enc, enc[1:]))


@pytest.mark.gpu
def test_quickpar_set_verifies_with_all_volumes(tmp_path):
    """repair.rs test_parser_loads_multiple_volumes: the intact QuickPar set,
    index and six volumes, verifies."""
    index = _qp_set(tmp_path)
    n, st = fmt.repair_ex(index, tmp_path, do_repair=False)
    assert n == 0 and st.damaged_blocks == 0 and st.recovery_blocks == 60


@pytest.mark.gpu
def test_repair_from_exponential_volumes(tmp_path):
    """robustness.rs test_exponential_volumes_many_blocks: 1 MB at 50 % in
    exponential volumes (several files), 200 KB overwritten, repaired."""
    files = make_files(tmp_path, [1_000_000], 33)
    orig = files[0].read_bytes()
    fmt.create(files, tmp_path / "volumes.par2", redundancy=50, scheme=fmt.SCHEME_EXPONENTIAL)
    assert len([p for p in tmp_path.iterdir() if p.suffix == ".par2"]) >= 3
    b = bytearray(orig)
    b[100_000:300_000] = b"\xff" * 200_000
    files[0].write_bytes(bytes(b))
    n, st = fmt.repair(tmp_path / "volumes.par2", tmp_path)
    assert n > 0 and files[0].read_bytes() == orig
