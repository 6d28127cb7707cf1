"""Host logic of the serving loop: what admission reserves per job (no GPU).
The reservation counts each job's outputs, bit planes (whole 2 KiB tiles),
coefficient records (96 bytes per input/output pair up to 24 outputs, 32
beyond) and, for a repair, its first pass's right-hand sides -- once each."""
import numpy as np

from par2gpu.serve import ServedJob


def test_create_job_reservation():
    src = np.zeros((100, 4096 + 64), np.uint8)
    j = ServedJob(0, "create", src, r=30)
    S = 4096 + 64
    assert j.scratch_bytes() == 30 * S + 100 * 3 * 2048 + 100 * 30 * 32


def test_small_repair_job_reservation():
    src = np.zeros((40, 8192), np.uint8)
    j = ServedJob(1, "repair", src, missing=np.array([2, 7, 9]), rec=np.zeros((3, 8192), np.uint8))
    # outputs + planes + 96-byte records + right-hand sides
    assert j.scratch_bytes() == 3 * 8192 + 40 * 8192 + 40 * 3 * 96 + 3 * 8192


def test_verify_job_reservation():
    src = np.zeros((500, 65536), np.uint8)
    assert ServedJob(2, "verify", src).scratch_bytes() == 500 * 20


def test_device_room_reads_free_memory_sparingly(monkeypatch):
    """Admission reads the device's free memory at most every 50 ms and
    counts the scratch of jobs admitted since the reading."""
    import torch

    from par2gpu.serve import _DeviceRoom

    reads = []

    def fake_mem_get_info(device):
        reads.append(device)
        return (3 << 30, 180 << 30)

    monkeypatch.setattr(torch.cuda, "mem_get_info", fake_mem_get_info)
    monkeypatch.setattr(torch.cuda, "memory_reserved", lambda device=None: 0)
    monkeypatch.setattr(torch.cuda, "memory_allocated", lambda device=None: 0)
    room = _DeviceRoom(every=0.05, margin=1 << 30)
    job = ServedJob(0, "create", np.zeros((2048, 1 << 20), np.uint8), r=1)  # 2 GiB of planes + 2 MB
    small = ServedJob(1, "create", np.zeros((64, 1 << 20), np.uint8), r=8)  # ~72 MiB
    assert not room.fits(job, 0.0)  # 2 GiB + 1 GiB margin > 3 GiB free
    assert room.fits(small, 0.01) and len(reads) == 1
    for _ in range(30):
        room.admitted(small)
    assert not room.fits(small, 0.02)  # 30 x 72 MiB counted against the reading
    assert room.fits(small, 0.2) and len(reads) == 2  # a fresh reading
