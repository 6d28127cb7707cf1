"""Python front end of libpar2gpu, the sm_100a GF(2^16) erasure-coding library.

The functions mirror the C ABI in include/par2gpu.h one to one (ctypes, no
torch types in the signatures).  Device buffers may be torch CUDA tensors,
whose data pointers are passed with ``device=True``.

There is no CPU fallback: loading fails loudly when the shared library is
missing, and every call raises ``Par2GpuError`` on a non-zero status.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libpar2gpu.so")

OK = 0
EINVAL = -1
ENOMEM = -2
ECUDA = -3
ESINGULAR = -4
ETIMEOUT = -5
ENODEV = -6
ERANGE = -7
ECANCELED = -8
DEVICE_PTRS = 0x1
PRIORITY_OPTIMAL = 40

_CODES = {EINVAL: "EINVAL", ENOMEM: "ENOMEM", ECUDA: "ECUDA", ESINGULAR: "ESINGULAR",
          ETIMEOUT: "ETIMEOUT", ENODEV: "ENODEV", ERANGE: "ERANGE", ECANCELED: "ECANCELED"}

# (name, restype, argtypes) of every exported entry point
_P = ctypes.c_void_p
_S = ctypes.c_size_t
_I = ctypes.c_int
_U32 = ctypes.c_uint32
_U16 = ctypes.c_uint16
SIGNATURES = [
    ("p2g_last_error", ctypes.c_char_p, []),
    ("p2g_create", _I, [_I, _P]),
    ("p2g_destroy", _I, [_P]),
    ("p2g_set_stream", _I, [_P, _P]),
    ("p2g_set_timing", _I, [_P, _I]),
    ("p2g_last_timing", _I, [_P, _P]),
    ("p2g_autotune", _I, [_P, _S, _S, _S, _I, _P]),
    ("p2g_set_plan", _I, [_P, _S, _S, _S, _P]),
    ("p2g_strategy_info", _I, [_P, _P, _P]),
    ("p2g_mul_slice", _I, [_P, _U16, _P, _S, _U32]),
    ("p2g_muladd", _I, [_P, _P, _P, _S, _U16, _U32]),
    ("p2g_muladd_region", _I, [_P, _P, _S, _P, _S, _P, _S, _S, _U32]),
    ("p2g_par2_constants", _I, [_S, _P]),
    ("p2g_encode", _I, [_P, _P, _S, _S, _P, _S, _P, _U32]),
    ("p2g_invert", _I, [_P, _S, _P, _P]),
    ("p2g_reconstruction_matrix", _I, [_P, _S, _P, _S, _P, _P]),
    ("p2g_repair", _I, [_P, _S, _S, _P, _S, _P, _P, _P, _P, _U32]),
    ("p2g_hash_slices", _I, [_P, _P, _S, _S, _P, _P, _U32]),
    ("p2g_verify_slices", _I, [_P, _P, _S, _S, _P, _P, _P, _U32]),
    ("p2g_encode_noalloc", _I, [_P, _P, _S, _S, _P, _S, _P]),
    ("p2g_supports_shuffle2x", _I, []),
    ("p2g_prepare_shuffle2x", _I, [_P, _P, _S]),
    ("p2g_muladd_shuffle2x", _I, [_P, _P, _P, _S, _U16]),
    ("p2g_muladd_region_shuffle2x", _I, [_P, _P, _S, _P, _S, _P, _S, _S]),
    ("p2g_finish_shuffle2x", _I, [_P, _P, _S]),
    ("p2g_batch_create", _I, [_P, _P, _S, _U32, _P]),
    ("p2g_batch_run", _I, [_P]),
    ("p2g_batch_launch", _I, [_P]),
    ("p2g_batch_poll", _I, [_P, _P]),
    ("p2g_batch_wait", _I, [_P]),
    ("p2g_batch_cancel", _I, [_P]),
    ("p2g_batch_destroy", _I, [_P]),
    ("p2g_batch_autotune", _I, [_P, _I, _P, _P]),
    ("p2g_batch_set_forms", _I, [_P, _P]),
]
JOB_CREATE, JOB_REPAIR, JOB_VERIFY = 1, 2, 3
# tile forms of the persistent batch kernel and the problem classes they are
# chosen for (par2gpu.h P2G_FORM_*, P2G_BATCH_CLASSES)
FORM_WIDE, FORM_SMALL, FORM_PAIRED = 0, 1, 2
BATCH_CLASSES = 8
BATCH_GRAPH = 0x2


class Job(ctypes.Structure):
    """p2g_job: one create / repair / verify job of a batch."""
    _fields_ = [("kind", _I), ("k", _S), ("slice_bytes", _S), ("col_begin", _S),
                ("col_end", _S), ("src", _P), ("n", _S), ("exps", _P), ("missing", _P),
                ("recovery", _P), ("inverse", _P), ("out", _P), ("md5_out", _P),
                ("crc_out", _P), ("status", _I)]
NOALLOC_SCRATCH_BYTES = 64 << 20
CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy: the legacy default stream


class Timing(ctypes.Structure):
    """p2g_timing: per-phase device milliseconds of the last call."""
    _fields_ = [("ms_records", ctypes.c_float), ("ms_planes", ctypes.c_float),
                ("ms_kernel", ctypes.c_float), ("ms_total", ctypes.c_float),
                ("launches", ctypes.c_int)]


class Plan(ctypes.Structure):
    """p2g_plan: tile shape of the multiply-accumulate kernel."""
    _fields_ = [("warps", ctypes.c_int), ("outputs_per_group", ctypes.c_int),
                ("warps_per_group", ctypes.c_int), ("output_blocks", ctypes.c_int),
                ("input_splits", ctypes.c_int), ("ms", ctypes.c_float),
                ("tile_symbols", ctypes.c_int), ("inputs_per_stage", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Par2GpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_CODES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libpar2gpu.so not built at {LIB_PATH}; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().p2g_last_error().decode(errors="replace")


def check(rc):
    if rc != OK:
        raise Par2GpuError(rc, last_error())
    return rc


def strategy_info():
    """(name, priority, available) as GaloisSimdStrategy::{name, priority,
    is_available} (par2-rs galois/simd/mod.rs:26-33)."""
    name = ctypes.c_char_p()
    prio = ctypes.c_int()
    avail = ctypes.c_int()
    check(lib().p2g_strategy_info(ctypes.byref(name), ctypes.byref(prio), ctypes.byref(avail)))
    return name.value.decode(), prio.value, bool(avail.value)


def par2_constants(k):
    out = np.zeros(k, np.uint16)
    check(lib().p2g_par2_constants(k, out.ctypes.data))
    return out


def encode_noalloc(stream, srcs, slice_bytes, exps, outs):
    """p2g_encode_noalloc: encode into caller device buffers with the library's
    fixed static scratch only (for callers that cannot allocate); enqueued on
    `stream` (an int cudaStream_t handle, 0 = default stream), not waited for."""
    e = np.ascontiguousarray(exps, np.uint32)
    check(lib().p2g_encode_noalloc(stream if stream else None, _ptr_array(srcs), len(srcs),
                                   slice_bytes,
                                   e.ctypes.data, len(e), _ptr_array(outs)))


def _ptr(x):
    """Address of a numpy array, a torch tensor or a raw int."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def _ptr_array(xs):
    """A C array of pointers: from a numpy uint64 array of addresses (used as
    is), from a 2-D array or tensor (one pointer per row, computed from its
    base and row stride), or from a list of ints / tensors / arrays."""
    if isinstance(xs, np.ndarray) and xs.dtype == np.uint64 and xs.ndim == 1:
        return _addr_param(np.ascontiguousarray(xs) if len(xs) else np.zeros(1, np.uint64))
    if isinstance(xs, np.ndarray) and xs.ndim == 2:
        return _row_addresses(xs.ctypes.data, xs.strides[0], xs.shape[0])
    if hasattr(xs, "data_ptr") and xs.dim() == 2:
        return _row_addresses(xs.data_ptr(), xs.stride(0) * xs.element_size(), xs.shape[0])
    arr = (ctypes.c_void_p * max(1, len(xs)))(*[_ptr(x) for x in xs])
    return arr


def _row_addresses(base, stride, n):
    if n == 0:
        return _addr_param(np.zeros(1, np.uint64))
    return _addr_param(np.uint64(base) + np.arange(n, dtype=np.uint64) * np.uint64(stride))


def _addr_param(a):
    # a void* argument over a uint64 address array; the pointer object holds
    # a reference to the array, so it lives until the call returns
    return a.ctypes.data_as(ctypes.c_void_p)


def _as_voidp(a):
    return a.ctypes.data if isinstance(a, np.ndarray) else ctypes.cast(a, ctypes.c_void_p)


class Context:
    """One p2g_ctx bound to a CUDA device (p2g_create / p2g_destroy)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(lib().p2g_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib().p2g_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        """Run on a caller CUDA stream: an int cudaStream_t handle such as
        torch's ``cuda_stream`` (0, the legacy default stream, is passed as
        cudaStreamLegacy); None restores the context's own stream."""
        if stream is None:
            check(lib().p2g_set_stream(self.h, None))
        else:
            check(lib().p2g_set_stream(self.h, stream if stream else CUDA_STREAM_LEGACY))

    def set_timing(self, enable=True):
        check(lib().p2g_set_timing(self.h, 1 if enable else 0))

    def last_timing(self):
        t = Timing()
        check(lib().p2g_last_timing(self.h, ctypes.byref(t)))
        return t

    def autotune(self, nin, nout, slice_bytes, reps=2):
        """Time the kernel's tile shapes for this problem shape and keep the
        fastest as this context's plan for it; returns the Plan."""
        p = Plan()
        check(lib().p2g_autotune(self.h, nin, nout, slice_bytes, reps, ctypes.byref(p)))
        return p

    def batch_autotune(self, reps=2):
        """Time the persistent batch kernel's tile forms per problem class and
        keep the fastest for this context's batches; returns (forms, ms), one
        entry per class (FORM_WIDE / FORM_SMALL / FORM_PAIRED)."""
        forms = np.zeros(BATCH_CLASSES, np.int32)
        ms = np.zeros(BATCH_CLASSES, np.float32)
        check(lib().p2g_batch_autotune(self.h, reps, forms.ctypes.data, ms.ctypes.data))
        return [int(f) for f in forms], [float(t) for t in ms]

    def batch_set_forms(self, forms=None):
        """Pin the batch kernel's form per class (None or -1: the heuristic)."""
        if forms is None:
            check(lib().p2g_batch_set_forms(self.h, None))
            return
        f = np.ascontiguousarray(forms, np.int32)
        if f.size != BATCH_CLASSES:
            raise ValueError(f"batch_set_forms takes {BATCH_CLASSES} forms")
        check(lib().p2g_batch_set_forms(self.h, f.ctypes.data))

    def set_plan(self, nin, nout, slice_bytes, warps, outputs_per_group, output_blocks,
                 input_splits=1, warps_per_group=1, tile_symbols=1024, inputs_per_stage=1):
        p = Plan(warps, outputs_per_group, warps_per_group, output_blocks, input_splits, 0.0,
                 tile_symbols, inputs_per_stage)
        check(lib().p2g_set_plan(self.h, nin, nout, slice_bytes, ctypes.byref(p)))

    # --- GaloisSimdStrategy mirror (galois/simd/mod.rs:36-58) -------------
    def mul_slice(self, scalar, data, device=False):
        n = data.numel() if hasattr(data, "numel") else data.size
        check(lib().p2g_mul_slice(self.h, scalar, _ptr(data), n, DEVICE_PTRS if device else 0))

    def muladd(self, dst, src, scalar, device=False):
        n = dst.numel() if hasattr(dst, "numel") else dst.size
        check(lib().p2g_muladd(self.h, _ptr(dst), _ptr(src), n, scalar,
                               DEVICE_PTRS if device else 0))

    def muladd_region(self, dsts, srcs, coeffs, region_offset, region_size, device=False):
        """dsts[d][off:off+len] ^= sum_s coeffs[d][s] * srcs[s][off:off+len]
        (u16 units); coeffs is a [ndst][nsrc] array."""
        co = np.ascontiguousarray(coeffs, np.uint16).reshape(len(dsts), len(srcs))
        rows = _ptr_array([co[d] for d in range(len(dsts))])
        check(lib().p2g_muladd_region(self.h, _ptr_array(dsts), len(dsts), _ptr_array(srcs),
                                      len(srcs), rows, region_offset, region_size,
                                      DEVICE_PTRS if device else 0))

    # --- the shuffle2x hooks (galois/simd/mod.rs:68-127) ------------------
    # Host u16 buffers (numpy uint16 arrays); between prepare and finish the
    # context holds a device copy of each and records the multiply-accumulates.
    def prepare_shuffle2x(self, buf):
        check(lib().p2g_prepare_shuffle2x(self.h, buf.ctypes.data, buf.size))

    def muladd_shuffle2x(self, dst, src, scalar):
        check(lib().p2g_muladd_shuffle2x(self.h, dst.ctypes.data, src.ctypes.data,
                                         min(dst.size, src.size), scalar))

    def muladd_region_shuffle2x(self, dsts, srcs, coeffs, region_offset, region_size):
        co = np.ascontiguousarray(coeffs, np.uint16).reshape(len(dsts), len(srcs))
        rows = _ptr_array([co[d] for d in range(len(dsts))])
        check(lib().p2g_muladd_region_shuffle2x(self.h, _ptr_array(dsts), len(dsts),
                                                _ptr_array(srcs), len(srcs), rows,
                                                region_offset, region_size))

    def finish_shuffle2x(self, buf):
        check(lib().p2g_finish_shuffle2x(self.h, buf.ctypes.data, buf.size))

    # --- coarse-grained encode (par2_rs.rs:687-902) -----------------------
    def encode(self, srcs, slice_bytes, exps, outs, device=False):
        e = np.ascontiguousarray(exps, np.uint32)
        check(lib().p2g_encode(self.h, _ptr_array(srcs), len(srcs), slice_bytes, e.ctypes.data,
                               len(e), _ptr_array(outs), DEVICE_PTRS if device else 0))

    def encode_array(self, src, exps):
        """Host convenience: src uint8 [k, S] -> recovery uint8 [r, S]."""
        src = np.ascontiguousarray(src, np.uint8)
        k, S = src.shape
        out = np.zeros((len(exps), S), np.uint8)
        self.encode(src, S, exps, out)
        return out

    # --- repair (par2_rs.rs:319-675) --------------------------------------
    def invert(self, A):
        """Exact GF(2^16) inverse of a square uint16 matrix (Par2GpuError with
        code ESINGULAR when it has none)."""
        A = np.ascontiguousarray(A, np.uint16)
        out = np.zeros_like(A)
        check(lib().p2g_invert(self.h, A.shape[0], A.ctypes.data, out.ctypes.data))
        return out

    def reconstruction_matrix(self, k, missing, exps):
        miss = np.ascontiguousarray(missing, np.uint64)
        e = np.ascontiguousarray(exps, np.uint32)
        out = np.zeros((len(miss), len(miss)), np.uint16)
        check(lib().p2g_reconstruction_matrix(self.h, k, miss.ctypes.data, len(miss),
                                              e.ctypes.data, out.ctypes.data))
        return out

    def repair(self, k, slice_bytes, missing, present, exps, recovery, outs, device=False):
        miss = np.ascontiguousarray(missing, np.uint64)
        e = np.ascontiguousarray(exps, np.uint32)
        check(lib().p2g_repair(self.h, k, slice_bytes, miss.ctypes.data, len(miss),
                               _ptr_array(present), e.ctypes.data, _ptr_array(recovery),
                               _ptr_array(outs), DEVICE_PTRS if device else 0))

    def repair_array(self, data, missing, exps, recovery):
        """Host convenience: data uint8 [k, S] (rows in `missing` ignored),
        recovery uint8 [m, S] -> rebuilt slices uint8 [m, S]."""
        data = np.ascontiguousarray(data, np.uint8)
        k, S = data.shape
        miss = sorted(int(x) for x in missing)
        mset = set(miss)
        present = [data[i] for i in range(k) if i not in mset]
        rec = np.ascontiguousarray(recovery, np.uint8)
        out = np.zeros((len(miss), S), np.uint8)
        self.repair(k, S, miss, present, exps, [rec[j] for j in range(len(miss))],
                    [out[j] for j in range(len(miss))])
        return out

    # --- per-slice MD5 + CRC32 (verify.rs:548-654, creator.rs:397-409) ----
    def hash_slices(self, slices, slice_bytes, device=False):
        n = len(slices)
        md5 = np.zeros((n, 16), np.uint8)
        crc = np.zeros(n, np.uint32)
        check(lib().p2g_hash_slices(self.h, _ptr_array(slices), n, slice_bytes, md5.ctypes.data,
                                    crc.ctypes.data, DEVICE_PTRS if device else 0))
        return md5, crc

    def verify_slices(self, slices, slice_bytes, md5_expect, crc_expect, device=False):
        n = len(slices)
        md5e = np.ascontiguousarray(md5_expect, np.uint8).reshape(n, 16)
        crce = np.ascontiguousarray(crc_expect, np.uint32)
        ok = np.zeros(n, np.uint8)
        check(lib().p2g_verify_slices(self.h, _ptr_array(slices), n, slice_bytes,
                                      md5e.ctypes.data, crce.ctypes.data, ok.ctypes.data,
                                      DEVICE_PTRS if device else 0))
        return ok.astype(bool)


class Batch:
    """A batch of jobs (p2g_batch_*).  Each job is a dict:
      create: kind=JOB_CREATE, k, slice_bytes, src (k device ptrs), exps, out (r ptrs)
      repair: kind=JOB_REPAIR, k, slice_bytes, src (k-m present ptrs), missing, exps,
              recovery (m ptrs), out (m ptrs), optional inverse (m x m uint16)
      verify: kind=JOB_VERIFY, k, slice_bytes, src (k ptrs) -> result md5 [k,16], crc [k]
    optional col_begin / col_end restrict create / repair to a byte range.
    Pointers are ints or torch CUDA tensors."""

    def __init__(self, ctx, jobs, graph=False):
        self.ctx = ctx
        self._keep = []
        self.jobs = (Job * max(1, len(jobs)))()
        self.specs = jobs
        self.results = []
        for j, spec in enumerate(jobs):
            J = self.jobs[j]
            J.kind = spec["kind"]
            J.k = spec["k"]
            J.slice_bytes = spec["slice_bytes"]
            J.col_begin = spec.get("col_begin", 0)
            J.col_end = spec.get("col_end", 0)
            src = _ptr_array(spec["src"])
            self._keep.append(src)
            J.src = _as_voidp(src)
            res = {}
            if spec["kind"] in (JOB_CREATE, JOB_REPAIR):
                e = np.ascontiguousarray(spec["exps"], np.uint32)
                out = _ptr_array(spec["out"])
                self._keep += [e, out]
                J.n = len(e)
                J.exps = e.ctypes.data
                J.out = _as_voidp(out)
            if spec["kind"] == JOB_REPAIR:
                miss = np.ascontiguousarray(spec["missing"], np.uint64)
                rec = _ptr_array(spec["recovery"])
                self._keep += [miss, rec]
                J.missing = miss.ctypes.data
                J.recovery = _as_voidp(rec)
                if spec.get("inverse") is not None:
                    inv = np.ascontiguousarray(spec["inverse"], np.uint16)
                    self._keep.append(inv)
                    J.inverse = inv.ctypes.data
            if spec["kind"] == JOB_VERIFY:
                res["md5"] = np.zeros((spec["k"], 16), np.uint8)
                res["crc"] = np.zeros(spec["k"], np.uint32)
                J.md5_out = res["md5"].ctypes.data
                J.crc_out = res["crc"].ctypes.data
            self.results.append(res)
        h = ctypes.c_void_p()
        check(lib().p2g_batch_create(ctx.h, ctypes.cast(self.jobs, ctypes.c_void_p), len(jobs),
                                     BATCH_GRAPH if graph else 0, ctypes.byref(h)))
        self.h = h

    def run(self):
        check(lib().p2g_batch_run(self.h))
        return [self.jobs[j].status for j in range(len(self.specs))]

    def launch(self):
        check(lib().p2g_batch_launch(self.h))

    def poll(self):
        d = ctypes.c_int()
        check(lib().p2g_batch_poll(self.h, ctypes.byref(d)))
        return bool(d.value)

    def wait(self):
        check(lib().p2g_batch_wait(self.h))
        return [self.jobs[j].status for j in range(len(self.specs))]

    def statuses(self):
        return [self.jobs[j].status for j in range(len(self.specs))]

    def cancel(self):
        """Stops a launched batch at its next work item (wait() then raises
        Par2GpuError with code ECANCELED)."""
        check(lib().p2g_batch_cancel(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().p2g_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
