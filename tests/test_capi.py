"""The C-ABI library loads without a GPU and exports every function the header declares."""
import ctypes
import os
import re

import pytest

from rqutils_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include',
                      'sqd_b200.h')


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    names = re.findall(r'\b(sqd_[a-z0-9_]+)\s*\(', text)
    return sorted(set(n for n in names if not n.endswith('_fn')))


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert b'sm_100a' in lib.sqd_version()


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIBPATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    names = set(declared_functions())
    bound = set(_lib.PROTOTYPES) | set(_lib.EXTRA_PROTOTYPES)
    assert names <= bound, sorted(names - bound)


def test_invalid_arguments_return_status_without_gpu():
    lib = _lib.load()
    out = ctypes.c_void_p()
    # num_qubits out of range is rejected before any CUDA call
    st = lib.sqd_paulis_create(None, None, None, None, 1, 0, 0, None, ctypes.byref(out), None)
    assert st == _lib.SQD_ERR_INVALID
    assert b'num_qubits' in lib.sqd_last_error()
    st = lib.sqd_space_create(None, 0, 8, 0, None, ctypes.byref(out))
    assert st == _lib.SQD_ERR_INVALID
    with pytest.raises(ValueError):
        _lib.check(st)


def header_enums():
    """name -> value for every `SQD_X = value` enumerator in the header."""
    text = re.sub(r'/\*.*?\*/', '', open(HEADER).read(), flags=re.S)
    return {m.group(1): int(m.group(2))
            for m in re.finditer(r'\b(SQD_[A-Z0-9_]+)\s*=\s*(-?\d+)', text)}


def test_python_constants_match_header_enums():
    enums = header_enums()
    for name in ('SQD_OK', 'SQD_ERR_INVALID', 'SQD_F64', 'SQD_C128', 'SQD_F32', 'SQD_C64',
                 'SQD_LOOKUP_HASH', 'SQD_LOOKUP_BSEARCH', 'SQD_LOOKUP_AUTO',
                 'SQD_LOOKUP_PRODUCT'):
        assert getattr(_lib, name) == enums[name], name
    from rqutils_b200.sqd import SQDOperator, _LOOKUPS
    assert SQDOperator.LAYOUTS == {'csr': enums['SQD_LAYOUT_CSR'],
                                   'product': enums['SQD_LAYOUT_PRODUCT'],
                                   'product-csr': enums['SQD_LAYOUT_PRODUCT_CSR']}
    assert _LOOKUPS['product'] == enums['SQD_LOOKUP_PRODUCT']
