"""ctypes front end of the C oracle (par2_oracle.c) and of the restated
par2-rs AVX2 strategy (cpu_simd_baseline.c).

TEST INFRASTRUCTURE ONLY -- see oracle/__init__.py.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_ORACLE = os.path.join(_BUILD, "libpar2oracle.so")
_CPUBASE = os.path.join(_BUILD, "libpar2cpubase.so")


def build():
    """Compile the oracle and the CPU baseline with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load(path):
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


_o = None
_b = None


def lib():
    global _o
    if _o is None:
        _o = _load(_ORACLE)
        P = ctypes.c_void_p
        S = ctypes.c_size_t
        _o.po_gf_mul.restype = ctypes.c_uint16
        _o.po_gf_mul.argtypes = [ctypes.c_uint16, ctypes.c_uint16]
        _o.po_gf_div.restype = ctypes.c_int
        _o.po_gf_div.argtypes = [ctypes.c_uint16, ctypes.c_uint16, P]
        _o.po_gf_pow.restype = ctypes.c_uint16
        _o.po_gf_pow.argtypes = [ctypes.c_uint16, ctypes.c_uint64]
        _o.po_par2_constants.argtypes = [S, P]
        _o.po_power_matrix.argtypes = [P, S, P, S, P]
        _o.po_encode.argtypes = [P, S, S, P, S, P]
        _o.po_muladd_region.argtypes = [P, S, P, S, P, S, S]
        _o.po_invert.restype = ctypes.c_int
        _o.po_invert.argtypes = [S, P, P]
        _o.po_reconstruct.restype = ctypes.c_int
        _o.po_reconstruct.argtypes = [S, S, P, S, P, P, P, P, ctypes.c_int, P]
        _o.po_md5.argtypes = [P, S, P]
        _o.po_crc32.restype = ctypes.c_uint32
        _o.po_crc32.argtypes = [P, S]
        _o.po_hash_slices.argtypes = [P, S, S, P, P]
        _o.po_calculate_block_size.restype = ctypes.c_uint64
        _o.po_calculate_block_size.argtypes = [ctypes.c_uint64]
        _o.po_recovery_count.restype = ctypes.c_uint64
        _o.po_recovery_count.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float]
    return _o


def cpubase():
    global _b
    if _b is None:
        _b = _load(_CPUBASE)
        P = ctypes.c_void_p
        S = ctypes.c_size_t
        _b.pb_encode.argtypes = [P, S, S, S, P, ctypes.c_int]
        _b.pb_muladd_region_split.argtypes = [P, S, P, S, P, S, ctypes.c_int]
        _b.pb_to_split.argtypes = [P, S]
        _b.pb_from_split.argtypes = [P, S]
    return _b


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def gf_mul(a, b):
    return int(lib().po_gf_mul(a, b))


def gf_div(a, b):
    out = ctypes.c_uint16(0)
    rc = lib().po_gf_div(a, b, ctypes.byref(out))
    return None if rc else int(out.value)


def gf_pow(a, n):
    return int(lib().po_gf_pow(a, n))


def par2_constants(k):
    out = np.zeros(k, np.uint16)
    lib().po_par2_constants(k, _p(out))
    return out


def power_matrix(bases, exps):
    """uint16 [len(exps), len(bases)]: bases[col] ** exps[row] in GF(2^16)."""
    b = np.ascontiguousarray(bases, np.uint16)
    e = np.ascontiguousarray(exps, np.uint32)
    out = np.zeros((len(e), len(b)), np.uint16)
    lib().po_power_matrix(_p(b), len(b), _p(e), len(e), _p(out))
    return out


def erasure_matrix(k, missing, exps):
    """A[row][col] = c_{missing[col]}^{exps[row]} with the PAR2 constants of k
    input slices (par2_rs.rs:346-353)."""
    return power_matrix(par2_constants(k)[np.asarray(missing)], exps)


def encode(src, exps):
    """src: uint8 [k, S] -> recovery uint8 [r, S] for the given exponents."""
    src = np.ascontiguousarray(src, np.uint8)
    k, S = src.shape
    exps = np.ascontiguousarray(exps, np.uint32)
    out = np.zeros((len(exps), S), np.uint8)
    lib().po_encode(_p(src), k, S, _p(exps), len(exps), _p(out))
    return out


def muladd_region(dsts, srcs, coeffs, off, length):
    """In-place dsts[d][off:off+len] ^= sum_s coeffs[d, s] * srcs[s][...] (u16)."""
    dp = (ctypes.c_void_p * len(dsts))(*[d.ctypes.data for d in dsts])
    sp = (ctypes.c_void_p * len(srcs))(*[s.ctypes.data for s in srcs])
    co = np.ascontiguousarray(coeffs, np.uint16)
    lib().po_muladd_region(ctypes.cast(dp, ctypes.c_void_p), len(dsts),
                           ctypes.cast(sp, ctypes.c_void_p), len(srcs), _p(co), off, length)


def invert(A):
    A = np.ascontiguousarray(A, np.uint16)
    m = A.shape[0]
    out = np.zeros_like(A)
    rc = lib().po_invert(m, _p(A), _p(out))
    return None if rc else out


def reconstruct(data, missing, rec_exps, rec, ref_row_quirk=False):
    """data uint8 [k, S] (missing rows ignored), missing sorted global indices,
    rec uint8 [m, S] with exponents rec_exps (lowest first).  Returns
    (out uint8 [m, S] or None when singular, number of moved rows)."""
    data = np.ascontiguousarray(data, np.uint8)
    k, S = data.shape
    miss = np.ascontiguousarray(missing, np.uint64)
    exps = np.ascontiguousarray(rec_exps, np.uint32)
    rec = np.ascontiguousarray(rec, np.uint8)
    m = len(miss)
    out = np.zeros((m, S), np.uint8)
    nsw = ctypes.c_uint64(0)
    rc = lib().po_reconstruct(k, S, _p(miss), m, _p(data), _p(exps), _p(rec), _p(out),
                              1 if ref_row_quirk else 0, ctypes.byref(nsw))
    return (None if rc else out), int(nsw.value)


def md5(buf):
    buf = np.ascontiguousarray(np.frombuffer(bytes(buf), np.uint8) if isinstance(buf, (bytes, bytearray)) else buf, np.uint8)
    out = np.zeros(16, np.uint8)
    lib().po_md5(_p(buf), buf.size, _p(out))
    return out.tobytes()


def crc32(buf):
    buf = np.ascontiguousarray(np.frombuffer(bytes(buf), np.uint8) if isinstance(buf, (bytes, bytearray)) else buf, np.uint8)
    return int(lib().po_crc32(_p(buf), buf.size))


def hash_slices(data):
    """data uint8 [n, S] -> (md5 uint8 [n, 16], crc uint32 [n])."""
    data = np.ascontiguousarray(data, np.uint8)
    n, S = data.shape
    md5s = np.zeros((n, 16), np.uint8)
    crcs = np.zeros(n, np.uint32)
    lib().po_hash_slices(_p(data), n, S, _p(md5s), _p(crcs))
    return md5s, crcs


def calculate_block_size(total):
    return int(lib().po_calculate_block_size(total))


def recovery_count(data_blocks, block_size, pct):
    return int(lib().po_recovery_count(data_blocks, block_size, pct))


def cpu_encode(src, r, nthreads):
    """The restated AVX2 strategy: recovery slices with exponents 0..r-1."""
    src = np.ascontiguousarray(src, np.uint8)
    k, S = src.shape
    out = np.zeros((r, S), np.uint8)
    cpubase().pb_encode(_p(src), k, S, r, _p(out), nthreads)
    return out


def cpu_muladd_region_split(dsts, srcs, coeffs, nthreads):
    """dsts/srcs: lists of uint8 arrays already in the split layout."""
    dp = (ctypes.c_void_p * len(dsts))(*[d.ctypes.data for d in dsts])
    sp = (ctypes.c_void_p * len(srcs))(*[s.ctypes.data for s in srcs])
    co = np.ascontiguousarray(coeffs, np.uint16)
    cpubase().pb_muladd_region_split(ctypes.cast(dp, ctypes.c_void_p), len(dsts),
                                     ctypes.cast(sp, ctypes.c_void_p), len(srcs), _p(co),
                                     dsts[0].size, nthreads)


def to_split(a):
    cpubase().pb_to_split(_p(a), a.size)


def from_split(a):
    cpubase().pb_from_split(_p(a), a.size)
