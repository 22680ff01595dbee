"""ctypes binding of the C ABI in include/ffbp_b200.h (the library fastsar_b200/libffbp_b200.so).

There is no fallback: a missing library, or a machine without a CUDA device, raises when a former is built."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libffbp_b200.so')

FFBP_OK, FFBP_E_ARG, FFBP_E_CUDA, FFBP_E_NOMEM, FFBP_E_WORKSPACE, FFBP_E_UNSUPPORTED = 0, -1, -2, -3, -4, -5
FFBP_E_TRANSFER = -6
PIX_AS_IS, PIX_POWER, PIX_SQUARE = 0, 1, 2          # ffbp_box_mean / ffbp_mean_add pixel kinds
FFBP_FINAL_FP32, FFBP_FINAL_TC_F16, FFBP_FINAL_TC_BF16X3 = 0, 1, 2
FFBP_LEVELS_TC = 0x100
KIND_NAMES = {1: 'amax', 2: 'level_fp32', 3: 'level_tc_gemm', 4: 'level_tc_fir', 5: 'final_fp32', 6: 'final_tc',
              7: 'level_tc'}
FFBP_KIND_LEVEL_TC_GEMM, FFBP_KIND_FINAL_TC, FFBP_KIND_LEVEL_TC = 3, 6, 7
FFBP_LEVELS_TC2 = 0x200

# every symbol include/ffbp_b200.h declares
EXPORTS = ('ffbp_last_error', 'ffbp_abi_version', 'ffbp_plan_create', 'ffbp_plan_destroy', 'ffbp_plan_workspace_bytes',
           'ffbp_form', 'ffbp_form_timed', 'ffbp_plan_info', 'ffbp_level', 'ffbp_phases', 'ffbp_final',
           'ffbp_bp_points_f64', 'ffbp_simulate', 'ffbp_form_static', 'ffbp_level_tc', 'ffbp_level_tc_scratch_bytes',
           'ffbp_form_profile', 'ffbp_exact_pad', 'ffbp_exact_backproject', 'ffbp_mlp_param_count',
           'ffbp_mlp_max_decimation', 'ffbp_mlp_work_bytes', 'ffbp_plan_host_bytes', 'ffbp_form_host', 'ffbp_gate_pad',
           'ffbp_gate_fold', 'ffbp_gate_taper', 'ffbp_batch_create', 'ffbp_batch_form', 'ffbp_batch_destroy', 'ffbp_mlp_taps', 'ffbp_mlp_grad', 'ffbp_mlp_train_step',
           'ffbp_plan_check', 'ffbp_plan_test_wait', 'ffbp_level_fused', 'ffbp_level_tc_ex', 'ffbp_plan_test_transfer',
           'ffbp_box_mean', 'ffbp_coherence', 'ffbp_multilook', 'ffbp_mean_add', 'ffbp_mean_image', 'ffbp_tile_stats',
           'ffbp_cross_spectrum', 'ffbp_ramp_multiply', 'ffbp_shift_crop', 'ffbp_window', 'ffbp_mosaic_pad', 'ffbp_mosaic_gather',
           'ffbp_mosaic_gate')

_c_int, _c_double, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p


class TcOpts(ctypes.Structure):
    """ffbp_tc_opts: launch options of a tensor-core level's first pass (0 keeps a field's default)."""
    _fields_ = [('nt', _c_int), ('sb', _c_int), ('copies', _c_int), ('repeat', _c_int), ('fir', _c_int),
                ('consumers', _c_int)]


class LevelDesc(ctypes.Structure):
    _fields_ = [('sx', _c_int), ('sy', _c_int), ('C', _c_int), ('Dk', _c_int), ('Dp', _c_int), ('K', _c_int),
                ('P', _c_int), ('Ko', _c_int), ('Po', _c_int),
                ('h_taps_k', _vp), ('Lk', _c_int), ('plk', _c_int),
                ('h_taps_p', _vp), ('Lp', _c_int), ('plp', _c_int),
                ('f0', _c_double), ('df', _c_double),
                ('h_ant', _vp), ('h_ref', _vp), ('h_cen', _vp), ('h_range', _vp), ('tc', TcOpts)]


class PlanDesc(ctypes.Structure):
    _fields_ = [('nlev', _c_int), ('levels', ctypes.POINTER(LevelDesc)), ('T', _c_int), ('nx', _c_int), ('ny', _c_int),
                ('Nx', _c_int), ('Ny', _c_int), ('ox', _c_int), ('oy', _c_int), ('spx', _c_double), ('spy', _c_double),
                ('e1', _c_double * 3), ('e2', _c_double * 3), ('Pf', _c_int), ('Qf', _c_int),
                ('f0f', _c_double), ('dff', _c_double), ('fcf', _c_double),
                ('h_ant_f', _vp), ('h_cen_f', _vp), ('h_first_f', _vp), ('h_wp', _vp), ('h_wk', _vp),
                ('h_wf', _vp), ('wf_ndim', _c_int), ('final_mode', _c_int), ('partial', _c_int)]


_LIB = None


def load():
    """The library, loaded once (built first when it is missing or older than its sources and nvcc is present)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    from . import build as _build
    if _build.stale():
        try:
            _build.build()
        except (OSError, RuntimeError) as e:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f'fastsar_b200: the CUDA library {LIB_PATH} is not built and could not be built '
                                   f'({e}); run python -m fastsar_b200.build on a machine with nvcc') from None
    L = ctypes.CDLL(LIB_PATH)
    L.ffbp_last_error.argtypes = [ctypes.c_char_p, _c_int]
    L.ffbp_abi_version.restype = _c_int
    L.ffbp_plan_create.argtypes = [ctypes.POINTER(PlanDesc), _vp, ctypes.POINTER(_vp)]
    L.ffbp_plan_destroy.argtypes = [_vp]
    L.ffbp_plan_workspace_bytes.argtypes = [_vp, ctypes.POINTER(ctypes.c_size_t)]
    L.ffbp_form.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp, ctypes.POINTER(_c_int)]
    L.ffbp_form_static.argtypes = [_vp, _vp, _vp, _vp, ctypes.POINTER(_c_int)]
    L.ffbp_plan_check.argtypes = [_vp, _vp]
    L.ffbp_plan_test_wait.argtypes = [_vp, _c_int, ctypes.c_uint]
    L.ffbp_plan_test_transfer.argtypes = [_vp, _c_int]
    L.ffbp_plan_host_bytes.argtypes = [_vp, ctypes.POINTER(ctypes.c_size_t)]
    L.ffbp_batch_create.argtypes = [ctypes.POINTER(_vp), _c_int, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                    ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t), _vp, ctypes.POINTER(_vp)]
    L.ffbp_batch_form.argtypes = [_vp, _vp, ctypes.POINTER(_c_int)]
    L.ffbp_batch_destroy.argtypes = [_vp]
    L.ffbp_gate_pad.argtypes = [_vp, _c_int, _c_int, _vp, _vp, _c_int, _c_int, _vp, _vp, _c_int, _vp]
    L.ffbp_gate_fold.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _vp]
    L.ffbp_gate_taper.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp]
    L.ffbp_form_host.argtypes = [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _c_int, _vp, ctypes.c_size_t, _vp,
                                 ctypes.c_size_t, _vp, ctypes.POINTER(_c_int)]
    L.ffbp_form_timed.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp, ctypes.POINTER(ctypes.c_float), _c_int]
    L.ffbp_plan_info.argtypes = [_vp, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)]
    L.ffbp_form_profile.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_size_t, _vp, ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(_c_int), _c_int]
    L.ffbp_level.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _c_double,
                             _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp]
    L.ffbp_level_tc.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                                _c_double, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t,
                                _vp, _vp]
    L.ffbp_level_tc_ex.argtypes = L.ffbp_level_tc.argtypes[:-1] + [ctypes.POINTER(TcOpts), _vp]
    L.ffbp_level_tc_scratch_bytes.argtypes = [_c_int, _c_int, _c_int, _c_int]
    L.ffbp_level_fused.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                                   _c_double, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp]
    L.ffbp_mlp_param_count.argtypes = []
    L.ffbp_mlp_work_bytes.argtypes = [_c_int]
    L.ffbp_mlp_taps.argtypes = [_vp, _vp, _c_int, _vp, _vp, _vp]
    L.ffbp_mlp_max_decimation.argtypes = []
    L.ffbp_mlp_grad.argtypes = [_vp, _vp, _c_int, _vp, ctypes.c_float, _vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _vp,
                                _vp, _vp]
    L.ffbp_mlp_train_step.argtypes = [_vp, _vp, _vp, _c_int, _vp, ctypes.c_float, _vp, _vp, _c_int, _vp, _vp, _c_int,
                                      ctypes.c_float, _c_int, _vp, _vp, _vp]
    L.ffbp_exact_pad.argtypes = [_vp, _c_int, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_int, _vp]
    L.ffbp_exact_backproject.argtypes = [_vp, _c_int, _c_int, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int,
                                         _c_int, _c_double, _c_double, _vp, _vp, _c_double, _c_double, _c_int, _c_int,
                                         _vp, _vp, _vp]
    L.ffbp_phases.argtypes = [_vp, _c_int, _vp, _c_int, _vp, _c_int, _vp, _c_double, _c_double, _c_int, _vp, _vp]
    L.ffbp_final.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _c_double, _c_double, _c_double,
                             _c_double, _vp, _vp, _vp, _c_double, _vp, _c_int, _vp, _vp]
    L.ffbp_bp_points_f64.argtypes = [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, ctypes.c_long, _c_double, _c_double, _vp,
                                     _vp]
    L.ffbp_simulate.argtypes = [_vp, _c_int, _c_int, _c_double, _c_double, _vp, _vp, _c_int, _vp, _vp]
    _f32, _long = ctypes.c_float, ctypes.c_long
    L.ffbp_box_mean.argtypes = [_vp, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp]
    L.ffbp_coherence.argtypes = [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp]
    L.ffbp_multilook.argtypes = [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp]
    L.ffbp_mean_add.argtypes = [_vp, _c_int, _long, _f32, _f32, _c_int, _vp, _vp, _vp]
    L.ffbp_mean_image.argtypes = [_vp, _vp, _long, _vp, _vp]
    L.ffbp_tile_stats.argtypes = [_vp, _c_int, _c_int, _c_int, _f32, _vp, _vp, _vp]
    L.ffbp_cross_spectrum.argtypes = [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp]
    L.ffbp_ramp_multiply.argtypes = [_vp, _c_int, _c_int, _vp, _vp, _vp]
    L.ffbp_window.argtypes = [_vp, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp]
    L.ffbp_shift_crop.argtypes = [_vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp]
    L.ffbp_mosaic_pad.argtypes = [_vp, _long, _c_int, _c_int, _c_int, _c_int, _vp, _c_double, _c_double, _vp, _vp]
    L.ffbp_mosaic_gather.argtypes = [_vp, _long, _c_int, _c_int, _c_int, _vp, _vp, _vp]
    L.ffbp_mosaic_gate.argtypes = [_vp, _long, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _c_double, _vp, _vp, _vp]
    for name in EXPORTS:
        getattr(L, name).restype = _c_int
    L.ffbp_level_tc_scratch_bytes.restype = ctypes.c_size_t
    L.ffbp_mlp_work_bytes.restype = ctypes.c_size_t
    _LIB = L
    return L


def last_error():
    L = load()
    buf = ctypes.create_string_buffer(2048)
    L.ffbp_last_error(buf, len(buf))
    return buf.value.decode(errors='replace')


def check(rc, what):
    """Raise the Python exception for a status code: ValueError for arguments and unsupported shapes, MemoryError
    for allocations, RuntimeError for CUDA failures."""
    if rc == FFBP_OK:
        return
    msg = f'{what}: {last_error()}'
    if rc in (FFBP_E_ARG, FFBP_E_UNSUPPORTED, FFBP_E_WORKSPACE):
        raise ValueError(msg)
    if rc == FFBP_E_NOMEM or 'out of memory' in msg:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def ptr(a):
    """Address of a numpy array's data (None for None)."""
    return None if a is None else a.ctypes.data


def tptr(t):
    """Address of a torch tensor's data (None for None)."""
    return None if t is None else t.data_ptr()


def c64(a):
    return np.ascontiguousarray(a, np.float64)


def c32(a):
    return np.ascontiguousarray(a, np.float32)
