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
