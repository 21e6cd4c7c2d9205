"""ctypes binding of the C ABI in ``include/sqd_b200.h`` (``rqutils_b200/lib/libsqd_b200.so``).

There is no CPU implementation behind this module: if the shared library is missing the import
of the product API fails, and every call that needs a GPU raises when CUDA is unavailable.
"""
import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, 'lib', 'libsqd_b200.so')

SQD_OK = 0
SQD_ERR_INVALID = -1
SQD_F64, SQD_C128, SQD_F32, SQD_C64 = 0, 1, 2, 3
SQD_PAULIS_FORCE_REAL = 1
SQD_LOOKUP_HASH, SQD_LOOKUP_BSEARCH, SQD_LOOKUP_AUTO, SQD_LOOKUP_PRODUCT = 0, 1, 2, 3
SQD_LOCG_FP64, SQD_LOCG_MIXED = 0, 1

_c = ctypes
_vp = _c.c_void_p
_i64 = _c.c_int64
_i32 = _c.c_int
_u32 = _c.c_uint32
_u64 = _c.c_uint64
_f64 = _c.c_double

MATVEC_FN = _c.CFUNCTYPE(_i32, _vp, _vp, _vp, _vp)

# name -> (restype, argtypes)
PROTOTYPES = {
    'sqd_version': (_c.c_char_p, []),
    'sqd_last_error': (_c.c_char_p, []),
    'sqd_paulis_create': (_i32, [_vp, _vp, _vp, _vp, _i64, _i32, _u32, _vp, _c.POINTER(_vp),
                                 _c.POINTER(_i32)]),
    'sqd_paulis_info': (_i32, [_vp, _c.POINTER(_i64), _c.POINTER(_i64), _c.POINTER(_i64),
                               _c.POINTER(_i32), _c.POINTER(_i32)]),
    'sqd_paulis_export': (_i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    'sqd_paulis_destroy': (None, [_vp]),
    'sqd_pack_states': (_i32, [_vp, _i64, _i32, _vp, _vp]),
    'sqd_space_create': (_i32, [_vp, _i64, _i32, _i64, _vp, _c.POINTER(_vp)]),
    'sqd_space_info': (_i32, [_vp, _c.POINTER(_i64), _c.POINTER(_i64), _c.POINTER(_i32),
                              _c.POINTER(_u64)]),
    'sqd_space_states': (_i32, [_vp, _vp, _vp]),
    'sqd_xsource': (_i32, [_vp, _u64, _i32, _vp, _vp]),
    'sqd_space_lookup': (_i32, [_vp, _vp, _i64, _i32, _vp, _vp]),
    'sqd_space_destroy': (None, [_vp]),
    'sqd_op_create': (_i32, [_vp, _vp, _i32, _i32, _i32, _vp, _c.POINTER(_vp)]),
    'sqd_op_info': (_i32, [_vp, _c.POINTER(_i64), _c.POINTER(_i64), _c.POINTER(_i32)]),
    'sqd_matvec': (_i32, [_vp, _vp, _vp, _i32, _vp]),
    'sqd_diagonal': (_i32, [_vp, _i64, _vp, _i32, _vp]),
    'sqd_vinit': (_i32, [_vp, _c.POINTER(_i64), _vp]),
    'sqd_op_csr': (_i32, [_vp, _vp, _vp, _vp, _vp]),
    'sqd_grad_terms': (_i32, [_vp, _vp, _vp, _i32, _vp, _vp]),
    'sqd_op_destroy': (None, [_vp]),
    'sqd_op_matvec_cb': (_i32, [_vp, _vp, _vp, _vp]),
    'sqd_locg': (_i32, [_i64, _i32, _vp, _vp, _vp, _i64, _c.POINTER(_vp), _i32, _f64, _i32,
                        _i32, _i32, _vp, _c.POINTER(_f64), _vp, _c.POINTER(_i32),
                        _c.POINTER(_f64)]),
    'sqd_eigenpair_small': (_i32, [_vp, _i64, _i32, _vp, _vp, _vp]),
    'sqd_locg_record': (_i32, [_vp, _i64, _c.POINTER(_i64)]),
}
# Library extensions beyond the header's core set (declared in the header as well).
EXTRA_PROTOTYPES = {
    'sqd_op_set_lanes': (_i32, [_vp, _i32, _i32]),
    'sqd_op_get_lanes': (_i32, [_vp, _i32, _c.POINTER(_i32)]),
    'sqd_vinit_noalloc': (_i32, [_vp, _c.POINTER(_i64), _vp]),
    'sqd_trim_memory': (_i32, [_u64]),
    'sqd_memory_stats': (_i32, [_c.POINTER(_u64), _c.POINTER(_u64), _c.POINTER(_u64), _i32]),
    'sqd_paulis_set_coeffs': (_i32, [_vp, _vp, _vp, _vp, _c.POINTER(_i32)]),
    'sqd_op_refresh': (_i32, [_vp, _vp]),
    'sqd_batch_create': (_i32, [_c.POINTER(_vp), _i32, _vp, _c.POINTER(_vp)]),
    'sqd_batch_info': (_i32, [_vp, _c.POINTER(_i64), _c.POINTER(_i64)]),
    'sqd_batch_set_lanes': (_i32, [_vp, _i32, _i32]),
    'sqd_batch_locg': (_i32, [_vp, _i32, _vp, _c.POINTER(_i64), _f64, _i32, _i32, _vp,
                              _c.POINTER(_f64), _vp, _c.POINTER(_i32), _c.POINTER(_f64)]),
    'sqd_batch_destroy': (None, [_vp]),
    'sqd_op_release_groups': (_i32, [_vp]),
    'sqd_op_cache_values': (_i32, [_vp, _vp]),
    'sqd_op_set_chunk': (_i32, [_vp, _i32, _i64]),
    'sqd_op_set_layout': (_i32, [_vp, _i32, _i32, _vp]),
    'sqd_op_get_layout': (_i32, [_vp, _i32, _c.POINTER(_i32)]),
    'sqd_op_product_info': (_i32, [_vp, _vp, _c.POINTER(_i64), _c.POINTER(_i64),
                                   _c.POINTER(_i64), _c.POINTER(_i64), _c.POINTER(_i64)]),
}


class SQDError(RuntimeError):
    """A failure reported by the CUDA library."""


_LIB = None


def load():
    """Load the shared library (once)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBPATH):
        raise ImportError(f'{LIBPATH} is missing: build it with rqutils_b200.build.build() '
                          '(or __graft_entry__.build())')
    lib = _c.CDLL(LIBPATH)
    for name, (res, args) in {**PROTOTYPES, **EXTRA_PROTOTYPES}.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(status):
    if status != SQD_OK:
        msg = load().sqd_last_error().decode(errors='replace')
        if status == SQD_ERR_INVALID:
            raise ValueError(msg)
        raise SQDError(f'sqd_b200 error {status}: {msg}')


def call(name, *args):
    check(getattr(load(), name)(*args))


def trim_memory(keep_bytes=0):
    """Return the library's cached device memory to the driver."""
    call('sqd_trim_memory', int(keep_bytes))


def memory_stats(reset_high=False):
    """(reserved, used, used_high) bytes of the library's memory pool on the current device."""
    vals = [_u64(0), _u64(0), _u64(0)]
    call('sqd_memory_stats', *(_c.byref(v) for v in vals), int(bool(reset_high)))
    return tuple(int(v.value) for v in vals)


def require_cuda():
    if not torch.cuda.is_available():
        raise SQDError('rqutils_b200 needs a CUDA GPU (sm_100a); no CPU fallback exists')


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return _vp(s.cuda_stream)


def ptr(t):
    return _vp(t.data_ptr()) if t is not None else _vp(0)


def dtype_code(dtype):
    return {torch.float64: SQD_F64, torch.complex128: SQD_C128, torch.float32: SQD_F32,
            torch.complex64: SQD_C64}[dtype]


def tensor_from_ptr(address, n, dtype, device):
    """Zero-copy 1-D CUDA tensor over device memory owned by the library or the caller."""
    real = {torch.float64: torch.float64, torch.complex128: torch.float64,
            torch.float32: torch.float32, torch.complex64: torch.float32}[dtype]
    per = 2 if dtype.is_complex else 1
    typestr = '<f8' if real == torch.float64 else '<f4'

    class _Iface:
        __cuda_array_interface__ = {'shape': (n * per,), 'typestr': typestr,
                                    'data': (int(address), False), 'version': 3,
                                    'strides': None}
    t = torch.as_tensor(_Iface(), device=device)
    return t.view(dtype) if dtype.is_complex else t
