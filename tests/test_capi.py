"""The C-ABI library on the CPU: it builds for sm_100a, loads, exports every symbol include/ffbp_b200.h declares, and
reports its ABI version and argument errors without touching a GPU."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    with open(os.path.join(ROOT, 'include', 'ffbp_b200.h')) as fh:
        src = fh.read()
    return sorted(set(re.findall(r'^\s*(?:int|size_t)\s+(ffbp_\w+)\s*\(', src, re.M)))


def test_header_declares_the_binding_exports():
    from fastsar_b200 import _lib
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_loads_and_exports_every_symbol():
    from fastsar_b200 import _lib
    L = _lib.load()
    for name in _declared():
        assert hasattr(L, name), name
    assert L.ffbp_abi_version() == 4


def test_argument_errors_without_a_gpu():
    from fastsar_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.ffbp_plan_create(None, None, ctypes.byref(h)) == _lib.FFBP_E_ARG
    assert 'null' in _lib.last_error()
    pd = _lib.PlanDesc()
    pd.nlev = 0
    assert L.ffbp_plan_create(ctypes.byref(pd), None, ctypes.byref(h)) == _lib.FFBP_E_ARG
    assert 'level' in _lib.last_error()
    assert L.ffbp_level(None, 1, 1, 1, None, 1, None, 0, 0, 1, 1, 0.0, None, 0, 0, 1, 1, None, None, None, None, None) == _lib.FFBP_E_ARG
    with pytest.raises(ValueError, match='ffbp_level'):
        _lib.check(_lib.FFBP_E_ARG, 'x')
