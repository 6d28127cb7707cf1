"""ctypes binding of include/par2format.h: create and repair of PAR2 sets
from files (Par2Creator::create, Par2Repairer::repair of par2-rs) with the
slices on the GPU.  Raises Par2FormatError with the library's message."""
import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lib",
                        "libpar2format.so")
OK, ERROR, ESINGULAR, EINSUFFICIENT, ECANCELLED, EDAMAGED = 0, -1, -4, -8, -9, -10
OP_SCANNING, OP_LOADING, OP_VERIFYING, OP_REPAIRING = 0, 1, 2, 3
PROGRESS_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64,
                               ctypes.c_uint64)
SCHEME_SINGLE, SCHEME_EXPONENTIAL = 0, 1


class Stats(ctypes.Structure):
    _fields_ = [("ms_scan", ctypes.c_double), ("ms_ingest", ctypes.c_double),
                ("ms_gpu", ctypes.c_double), ("ms_write", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("block_size", ctypes.c_uint64),
                ("data_blocks", ctypes.c_uint64), ("recovery_blocks", ctypes.c_uint64),
                ("bytes_read", ctypes.c_uint64), ("damaged_blocks", ctypes.c_uint64),
                ("files_written", ctypes.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


SIGNATURES = [
    ("p2f_create", [ctypes.POINTER(ctypes.c_char_p), ctypes.c_size_t, ctypes.c_char_p,
                    ctypes.c_uint64, ctypes.c_float, ctypes.c_int, ctypes.POINTER(Stats)]),
    ("p2f_create_ex", [ctypes.POINTER(ctypes.c_char_p), ctypes.c_size_t, ctypes.c_char_p,
                       ctypes.c_uint64, ctypes.c_float, ctypes.c_int, PROGRESS_FN,
                       ctypes.c_void_p, ctypes.POINTER(Stats)]),
    ("p2f_repair", [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64),
                    ctypes.POINTER(Stats)]),
    ("p2f_repair_ex", [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, PROGRESS_FN,
                       ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                       ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Stats)]),
    ("p2f_streaming_encode", [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                              ctypes.c_void_p, ctypes.c_int]),
    ("p2f_last_error", []),
]

_lib = None


class Par2FormatError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (code {code})")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        from . import lib as gpu_lib

        gpu_lib()  # libpar2gpu.so first: libpar2format.so links against it
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_char_p if name == "p2f_last_error" else ctypes.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != OK:
        raise Par2FormatError(rc, lib().p2f_last_error().decode())


def create(inputs, output=None, block_size=0, redundancy=5.0, scheme=SCHEME_EXPONENTIAL,
           progress=None):
    """Writes the set of `inputs` (paths); returns the call's Stats.
    progress(operation, current, total), if given, receives the encoding
    progress (p2f_create_ex) on this thread."""
    arr = (ctypes.c_char_p * len(inputs))(*[os.fsencode(str(p)) for p in inputs])
    st = Stats()
    out = os.fsencode(str(output)) if output else None
    if progress is None:
        _check(lib().p2f_create(arr, len(inputs), out, block_size, redundancy, scheme,
                                ctypes.byref(st)))
    else:
        cb = PROGRESS_FN(lambda user, op, cur, tot: progress(op, cur, tot))
        _check(lib().p2f_create_ex(arr, len(inputs), out, block_size, redundancy, scheme, cb,
                                   None, ctypes.byref(st)))
    return st


def repair(par2_path, directory):
    """Verifies and repairs the set's files in `directory`; returns
    (slices rebuilt, Stats)."""
    n = ctypes.c_uint64()
    st = Stats()
    _check(lib().p2f_repair(os.fsencode(str(par2_path)), os.fsencode(str(directory)),
                            ctypes.byref(n), ctypes.byref(st)))
    return n.value, st


def repair_ex(par2_path, directory, do_repair=True, purge=False, progress=None, cancel=None):
    """repair_with_callbacks_cancellable: progress(operation, current, total)
    is called on this thread; `cancel` is a ctypes.c_int32 another thread may
    set non-zero.  Returns (slices rebuilt, Stats)."""
    cb = PROGRESS_FN(lambda user, op, cur, tot: progress(op, cur, tot)) if progress \
        else PROGRESS_FN()
    n = ctypes.c_uint64()
    st = Stats()
    _check(lib().p2f_repair_ex(os.fsencode(str(par2_path)), os.fsencode(str(directory)),
                               int(bool(do_repair)), int(bool(purge)), cb, None,
                               ctypes.byref(cancel) if cancel is not None else None,
                               ctypes.byref(n), ctypes.byref(st)))
    return n.value, st


def streaming_encode(src, r, threads=0):
    """par2-rs's streaming encoder path over the strategy interface
    (p2f_streaming_encode): src uint8 [k, S] host array -> recovery slices
    uint8 [r, S] with exponents 0..r-1."""
    import numpy as np

    src = np.ascontiguousarray(src, np.uint8)
    k, S = src.shape
    out = np.zeros((r, S), np.uint8)
    sp = (np.uint64(src.ctypes.data) + np.arange(k, dtype=np.uint64) * np.uint64(S)) if k \
        else np.zeros(1, np.uint64)
    op = (np.uint64(out.ctypes.data) + np.arange(r, dtype=np.uint64) * np.uint64(S)) if r \
        else np.zeros(1, np.uint64)
    _check(lib().p2f_streaming_encode(sp.ctypes.data, k, S, r, op.ctypes.data, threads))
    return out
