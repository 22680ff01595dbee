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
    assert L.ffbp_abi_version() == 5


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


def test_stack_product_argument_errors_without_a_gpu():
    from fastsar_b200 import _lib
    L = _lib.load()
    p = ctypes.c_void_p(256)          # never dereferenced: each call below fails its argument checks first
    E, U = _lib.FFBP_E_ARG, _lib.FFBP_E_UNSUPPORTED
    assert L.ffbp_box_mean(None, 1, 4, 4, 5, 0, p, None) == E
    assert L.ffbp_box_mean(p, 3, 4, 4, 5, 0, p, None) == E
    assert L.ffbp_box_mean(p, 1, 4, 4, 34, 0, p, None) == U and '33' in _lib.last_error()
    assert L.ffbp_box_mean(p, 1, 0, 4, 5, 0, p, None) == E
    assert L.ffbp_coherence(p, p, 4, 4, 5, 65, p, None) == U
    assert L.ffbp_coherence(p, None, 4, 4, 5, 5, p, None) == E
    assert L.ffbp_multilook(p, None, 4, 4, 0, 1, p, None) == E
    assert L.ffbp_mean_add(p, 0, 16, 1.0, 1.0, 1, p, p, None) == E
    assert L.ffbp_tile_stats(p, 64, 64, 0, 1.0, p, p, None) == E
    assert L.ffbp_cross_spectrum(p, p, 1, 4, 3, 1, p, None, p, p, None) == E
    assert L.ffbp_cross_spectrum(p, p, 0, 4, 3, 1, None, None, p, p, None) == E
    assert L.ffbp_shift_crop(p, 2, p, 1, 4, 4, 0, 0, p, None) == E and 'leading' in _lib.last_error()
    assert L.ffbp_window(p, 0, 4, 4, p, p, p, p, None) == E
    assert L.ffbp_window(p, 1, 4, 4, None, p, p, p, None) == E
