"""Pointer tables of the ctypes binding (no GPU needed): every form a slice
table may take turns into the same row addresses."""
import ctypes

import numpy as np
import torch

import par2gpu


def _addresses(param, n):
    return [int(x) for x in ctypes.cast(param, ctypes.POINTER(ctypes.c_uint64))[:n]]


def test_2d_numpy_rows():
    a = np.zeros((37, 96), np.uint8)[:, 16:]
    assert _addresses(par2gpu._ptr_array(a), 37) == [a[i].ctypes.data for i in range(37)]


def test_2d_tensor_rows():
    t = torch.zeros((9, 40), dtype=torch.uint8)[:, 8:]
    assert _addresses(par2gpu._ptr_array(t), 9) == [t[i].data_ptr() for i in range(9)]


def test_list_and_uint64_forms_agree():
    a = np.zeros((5, 64), np.uint8)
    rows = [a[i] for i in range(5)]
    want = [r.ctypes.data for r in rows]
    assert _addresses(par2gpu._ptr_array(rows), 5) == want
    assert _addresses(par2gpu._ptr_array(np.array(want, np.uint64)), 5) == want
    assert _addresses(par2gpu._ptr_array(want), 5) == want


def test_empty_tables_are_valid_pointers():
    for xs in ([], np.zeros((0, 8), np.uint8), np.zeros(0, np.uint64)):
        assert ctypes.cast(par2gpu._ptr_array(xs), ctypes.c_void_p).value
