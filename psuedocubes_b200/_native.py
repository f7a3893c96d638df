"""ctypes binding of libpcube (include/pcube.h) and the status-code to exception mapping.

The library is built in-tree by ``psuedocubes_b200.build`` into ``psuedocubes_b200/_lib``.  There
is no fallback: if the shared library is missing or cannot be loaded, every device operation
raises ``RuntimeError`` naming the missing file.
"""
from __future__ import annotations

import ctypes
import hashlib
import time
import weakref
from functools import lru_cache
from pathlib import Path
from typing import Any

import numpy as np

LIB_DIR = Path(__file__).resolve().parent / '_lib'
LIB_PATH = LIB_DIR / 'libpcube.so'

PC_OK, PC_OVERFLOW, PC_INVALID, PC_ARITHMETIC, PC_TIMEOUT, PC_NOMEM, PC_CUDA = range(7)

#: Every symbol include/pcube.h declares.
SYMBOLS = ('pc_version', 'pc_device_count', 'pc_last_error', 'pc_init', 'pc_free', 'pc_mem_info', 'pc_copy_info',
           'pc_host_alloc', 'pc_host_free',
           'pc_device_info', 'pc_sync', 'pc_mark', 'pc_elapsed', 'pc_buf_upload', 'pc_buf_download', 'pc_buf_size', 'pc_buf_free',
           'pc_buf_searchsorted', 'pc_focus_create', 'pc_focus_free', 'pc_focus_info', 'pc_focus_window',
           'pc_filters_create', 'pc_filters_free', 'pc_run_batch', 'pc_run_lease', 'pc_run_leases', 'pc_multi_create',
           'pc_multi_run', 'pc_multi_layout', 'pc_multi_results', 'pc_multi_free', 'pc_run_plain',
           'pc_run_plain_static', 'pc_scopes_json', 'pc_cube_roots', 'pc_selftest_wide')

PC_RUN_GRAPH = 1


class Tuning(ctypes.Structure):
    _fields_ = [('bitset_filters', ctypes.c_uint32), ('block_words', ctypes.c_uint32),
                ('words_per_thread', ctypes.c_uint32), ('v_chunk', ctypes.c_uint32),
                ('threads', ctypes.c_uint32), ('deep_records', ctypes.c_uint32), ('reserved', ctypes.c_uint32 * 2)]


class Stats(ctypes.Structure):
    _fields_ = [('kernel_ms', ctypes.c_double), ('bounds_ms', ctypes.c_double), ('window_ms', ctypes.c_double),
                ('total_ms', ctypes.c_double), ('work_items', ctypes.c_uint64), ('outputs', ctypes.c_uint64),
                ('launches', ctypes.c_uint64), ('reserved', ctypes.c_uint64 * 5), ('h2d_bytes', ctypes.c_uint64),
                ('d2h_bytes', ctypes.c_uint64)]

    def as_dict(self) -> dict[str, Any]:
        return dict(kernel_ms=self.kernel_ms, bounds_ms=self.bounds_ms, window_ms=self.window_ms,
                    total_ms=self.total_ms, outputs=int(self.outputs), launches=int(self.launches),
                    h2d_bytes=int(self.h2d_bytes), d2h_bytes=int(self.d2h_bytes),
                    deep_survivors=int(self.work_items), bitset_filters=int(self.reserved[0]),
                    block_words=int(self.reserved[1]), threads=int(self.reserved[2]),
                    cheap_filters=int(self.reserved[3]), graph=bool(self.reserved[4]))


class Window(ctypes.Structure):
    """One window of a multi-window launch (pc_window)."""
    _fields_ = [('first', ctypes.c_uint64), ('end', ctypes.c_uint64), ('width', ctypes.c_uint64),
                ('lo0', ctypes.c_uint64), ('lo1', ctypes.c_uint64), ('hi0', ctypes.c_uint64), ('hi1', ctypes.c_uint64),
                ('focus_a', ctypes.c_uint32), ('focus_b', ctypes.c_uint32), ('family', ctypes.c_uint32),
                ('reserved', ctypes.c_uint32)]


_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_U64P = np.ctypeslib.ndpointer(dtype=np.uint64, flags='C_CONTIGUOUS')
_U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags='C_CONTIGUOUS')
_U8P = np.ctypeslib.ndpointer(dtype=np.uint8, flags='C_CONTIGUOUS')


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    """Load libpcube.so; raise if it is absent (no CPU path exists)."""
    if not LIB_PATH.exists():
        raise RuntimeError(f'libpcube is not built: {LIB_PATH} is missing; run psuedocubes_b200.build.build()')
    so = ctypes.CDLL(str(LIB_PATH))
    pp = ctypes.POINTER(_P)
    so.pc_version.restype = ctypes.c_int
    so.pc_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    so.pc_last_error.argtypes = [_P]
    so.pc_last_error.restype = ctypes.c_char_p
    so.pc_init.argtypes = [ctypes.c_int, _U64, ctypes.c_double, pp]
    so.pc_free.argtypes = [_P]
    so.pc_mem_info.argtypes = [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64), ctypes.POINTER(_U64)]
    so.pc_copy_info.argtypes = [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]
    so.pc_device_info.argtypes = [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_int]
    so.pc_sync.argtypes = [_P]
    so.pc_mark.argtypes = [_P, ctypes.c_int]
    so.pc_elapsed.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    so.pc_buf_upload.argtypes = [_P, _U64P, _U64, pp]
    so.pc_buf_download.argtypes = [_P, _P, _U64, _U64, _U64P]
    so.pc_buf_size.argtypes = [_P, ctypes.POINTER(_U64)]
    so.pc_buf_free.argtypes = [_P, _P]
    so.pc_buf_searchsorted.argtypes = [_P, _P, _U64P, _U64, _U64P]
    so.pc_focus_create.argtypes = [_P, _U64, _U32, _U32P, _U32P, _U32P, _U64, pp]
    so.pc_focus_free.argtypes = [_P, _P]
    so.pc_focus_info.argtypes = [_P, _U64P]
    so.pc_focus_window.argtypes = [_P, _P, _U64, _U64, _U64, pp, ctypes.POINTER(_U64)]
    so.pc_filters_create.argtypes = [_P, _U64, _U64, _U32P, _U32, _U8P, pp]
    so.pc_filters_free.argtypes = [_P, _P]
    so.pc_run_batch.argtypes = [_P, _P, ctypes.POINTER(Tuning), _P, _U64, _U64, _P, _U64, _U64,
                                _U64, _U64, _U64, _U64, _U64, _U64, _U32, _U64,
                                _U64P, _U64P, _U64P, _U64, ctypes.POINTER(_U64), ctypes.POINTER(Stats)]
    so.pc_run_lease.argtypes = [_P, _P, _P, _P, ctypes.POINTER(Tuning), _U64, _U64, _U64,
                                _U64, _U64, _U64, _U64, _U64P, _U64P, _U64P, _U64, ctypes.POINTER(_U64),
                                ctypes.POINTER(Stats)]
    so.pc_multi_create.argtypes = [_P, ctypes.POINTER(_P), _U32, ctypes.POINTER(_P), _U32, ctypes.POINTER(Window), _U32,
                                   ctypes.POINTER(Tuning), _U64, pp]
    so.pc_multi_run.argtypes = [_P, _P, _U32, ctypes.POINTER(Stats)]
    so.pc_multi_layout.argtypes = [_P, _U32P, _U64P, _U64P]
    so.pc_multi_results.argtypes = [_P, _P, _U64P, _U64P, _U64P, _U64, ctypes.POINTER(_U64)]
    so.pc_multi_free.argtypes = [_P, _P]
    so.pc_run_plain.argtypes = [_P, _P, _P, _U64, _U64, _P, _U64, _U64, _U64, _U64, _U64, _U64,
                                _U64P, _U64P, _U64, ctypes.POINTER(Stats)]
    so.pc_run_plain_static.argtypes = [ctypes.c_int, _U64P, _U64, _U64P, _U64, _U64, _U64, _U64, _U64, _U64, _U64,
                                       _U32P, _U32, _U8P, _U64P, _U64P, _U64, ctypes.c_char_p, ctypes.c_int]
    so.pc_scopes_json.argtypes = [_U64P, _U32, _U32, _U64, _U64, _U64, _U64, _U32, ctypes.c_char_p, ctypes.c_void_p,
                                  _U64, ctypes.POINTER(_U64)]
    so.pc_run_leases.argtypes = [_P, _P, _P, _P, ctypes.POINTER(Tuning), _U32, _U64P, _U64P, _U64, _U64, _U64, _U64, _U64,
                                 pp, pp, pp, _U64, _U64P, ctypes.POINTER(Stats),
                                 np.ctypeslib.ndpointer(dtype=np.int32, flags='C_CONTIGUOUS')]
    so.pc_host_alloc.argtypes = [_U64, ctypes.POINTER(_P)]
    so.pc_host_free.argtypes = [_P]
    so.pc_cube_roots.argtypes = [_P, _U64, _U64, _U32, ctypes.c_void_p, _U64, ctypes.POINTER(_U64),
                                 ctypes.POINTER(ctypes.c_double)]
    so.pc_selftest_wide.argtypes = [_P, _U64P, _U64P, _U64]
    return so


def library_record() -> dict[str, Any]:
    """Identity of the loaded kernels (the reference records one entry per NVRTC compile)."""
    started = time.perf_counter()
    data = LIB_PATH.read_bytes()
    lib()
    return dict(name='libpcube', source_sha256=hashlib.sha256(data).hexdigest(),
                wall_seconds=time.perf_counter() - started, registers=None, local_bytes=None,
                shared_bytes=None, arch='sm_100a')


def raise_for(code: int, ctx: Any = None, what: str = '') -> None:
    """Map a libpcube status to the reference's exception types."""
    if code == PC_OK:
        return
    message = ''
    if ctx:
        raw = lib().pc_last_error(ctx)
        message = raw.decode() if raw else ''
    message = message or what or f'libpcube status {code}'
    if code == PC_OVERFLOW:
        raise OverflowError(message)
    if code == PC_INVALID:
        raise ValueError(message)
    if code == PC_ARITHMETIC:
        raise ArithmeticError(message)
    if code == PC_TIMEOUT:
        raise TimeoutError('BUDGET_EXHAUSTED')
    if code == PC_NOMEM:
        raise MemoryError(message)
    raise RuntimeError(f'CUDA failure in libpcube: {message}')


def pinned(count: int, dtype: Any = np.uint64) -> np.ndarray:
    """A zeroed numpy array in page-locked host memory (pc_host_alloc), freed with the array; the
    library copies results into such buffers at full link speed."""
    dtype = np.dtype(dtype)
    nbytes = max(1, int(count)) * dtype.itemsize
    ptr = _P()
    so = lib()
    raise_for(so.pc_host_alloc(nbytes, ctypes.byref(ptr)), None, 'page-locked host buffer')
    raw = (ctypes.c_uint8 * nbytes).from_address(ptr.value)
    array = np.frombuffer(raw, dtype=np.uint8).view(dtype)[:max(0, int(count))]
    array[:] = 0
    weakref.finalize(raw, so.pc_host_free, ptr.value)
    return array


def device_count() -> int:
    n = ctypes.c_int(0)
    lib().pc_device_count(ctypes.byref(n))
    return n.value


def u64(a: Any) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)
