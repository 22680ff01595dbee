"""The former surface of the reference (fastsar/api.py): ImageFormer and form_image, on the B200.

    former = ImageFormer(ant, fmin, df, K, nx, ny, spx, spy, e1, e2)     # plan + device geometry, once per geometry
    img = former(S)                                                      # S [P, K] complex -> complex64 [nx, ny]
    img = form_image(S, ant, fmin, df, nx, ny, spx, spy, e1, e2)         # one call (plans every time)

Same arguments, defaults, conventions and errors as the reference's (fastsar/api.py:312-716): pixel (i, j) sits at
(i - nx/2) spx e1 + (j - ny/2) spy e2 about the scene reference point; the history follows the CPHD convention
exp(-j 4 pi f dR / c); a Taylor window (-35 dB, nbar 4) is applied unless window=False; T='auto' picks the largest
final tile (32 or 16) whose predicted error meets target_db. The planner is fastsar_b200.plan (the reference's,
restated); the formation runs in the CUDA library (fastsar_b200/libffbp_b200.so) through its C ABI
(include/ffbp_b200.h), with device memory and streams from PyTorch.

Backends: 'auto' and 'cuda' run on the GPU. There is no CPU, JAX or TPU path in this package; asking for one raises
ValueError, as the reference does for a backend its machine lacks.

Precision: 'float32' (default): float32 arithmetic everywhere, the final stage on the CUDA cores or, where built,
as three bfloat16 products on the tensor cores (the reference's float32 CUDA default, fastsar/ffbp_cuda.py:949-953);
FASTSAR_FINAL=fp32 keeps the CUDA cores. 'float16': the final stage's operands in float16 on the tensor cores with
float32 accumulation (T = 16 or 32).
"""
import ctypes
import os
import warnings

import numpy as np

from . import _lib
from . import plan as _plan
from .sim import Collect

C = 299792458.0
BACKENDS = ('auto', 'tpu', 'cuda', 'cpu', 'jax', 'metal')


def _window(P, K, sll=35.0, nbar=4):
    """The Taylor windows over pulses and samples, float32 (fastsar/api.py:54-56)."""
    from scipy.signal.windows import taylor
    return (taylor(P, nbar=nbar, sll=sll, norm=False).astype(np.float32),
            taylor(K, nbar=nbar, sll=sll, norm=False).astype(np.float32))


def _backend(backend):
    if backend not in BACKENDS:
        raise ValueError(f'unknown backend {backend!r}: one of {", ".join(map(repr, BACKENDS))}')
    if backend not in ('auto', 'cuda'):
        raise ValueError(f"backend {backend!r} is not part of fastsar_b200, which forms images on the GPU only "
                         "(backend='auto' or 'cuda')")
    import torch
    if not torch.cuda.is_available():
        raise ValueError("backend 'cuda' needs an NVIDIA GPU; this machine has none")
    return 'cuda'


def _check_history(S, P=None, name='phase history'):
    """S [P, K] complex with at least 2 pulses and 2 samples (fastsar/api.py:132-152; the scan for NaN and inf runs
    on the device, in the first level)."""
    if not hasattr(S, 'ndim'):
        S = np.asarray(S)
    if S.ndim != 2:
        raise ValueError(f'{name} must be 2-D [pulses, samples], got shape {tuple(S.shape)}')
    kind = S.dtype.kind if isinstance(S, np.ndarray) else ('c' if S.is_complex() else 'f')
    if kind != 'c':
        raise TypeError(f'{name} must be complex (complex64 or complex128), got {S.dtype}')
    if P is not None and S.shape[0] != P:
        raise ValueError(f'{name} has {S.shape[0]} pulses but there are {P} antenna positions')
    if S.shape[0] < 2 or S.shape[1] < 2:
        raise ValueError(f'{name} needs at least 2 pulses and 2 samples, got shape {tuple(S.shape)}')
    return S


def _check_positions(a, name='antenna positions', P=None):
    """a [P, 3] finite float64 with at least 2 rows (fastsar/api.py:155-166)."""
    a = np.asarray(a, np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError(f'{name} must be [pulses, 3], got shape {a.shape}')
    if P is not None and len(a) != P:
        raise ValueError(f'{name}: {len(a)} rows for {P} pulses')
    if len(a) < 2:
        raise ValueError(f'{name}: at least 2 pulses are needed, got {len(a)}')
    if not np.isfinite(a).all():
        raise ValueError(f'{name}: non-finite values (NaN or inf)')
    return a


def _check_grid(nx, ny, spx, spy, e1, e2):
    """Positive integer pixel counts, positive spacings and orthonormal axes (fastsar/api.py:169-183)."""
    for n, v in (('nx', nx), ('ny', ny)):
        if np.ndim(v) != 0 or not np.isfinite(v) or v < 1 or int(v) != v:
            raise ValueError(f'{n} must be a positive integer, got {v!r}')
    for n, v in (('spx', spx), ('spy', spy)):
        if not np.isfinite(v) or v <= 0:
            raise ValueError(f'{n} must be a positive spacing in meters, got {v!r}')
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    if e1.shape != (3,) or e2.shape != (3,):
        raise ValueError(f'e1 and e2 must be 3-vectors, got shapes {e1.shape} and {e2.shape}')
    if abs(e1 @ e1 - 1) > 1e-6 or abs(e2 @ e2 - 1) > 1e-6 or abs(e1 @ e2) > 1e-6:
        raise ValueError(f'e1 and e2 must be orthonormal (unit length, perpendicular), got {e1.tolist()} and {e2.tolist()}')
    return int(nx), int(ny), e1, e2


def _final_mode(precision):
    """The formation mode of a precision: 'float32' the float32 kernels (FASTSAR_FINAL=tc3 puts the final stage on
    the tensor cores in split bfloat16); 'float16' the levels and the final stage on the tensor cores, the levels in
    two passes through a float16 intermediate (FASTSAR_LEVELS=tc1: in one pass; fp32: on the float32 kernel)."""
    if precision == 'float16':
        lv = os.environ.get('FASTSAR_LEVELS', 'tc').strip().lower() or 'tc'
        if lv not in ('tc', 'tc1', 'tc2', 'fp32'):
            raise ValueError(f"FASTSAR_LEVELS must be 'tc', 'tc1', 'tc2' or 'fp32', got {lv!r}")
        flags = {'tc': _lib.FFBP_LEVELS_TC | _lib.FFBP_LEVELS_TC2, 'tc1': _lib.FFBP_LEVELS_TC,
                 'tc2': _lib.FFBP_LEVELS_TC | _lib.FFBP_LEVELS_TC2, 'fp32': 0}[lv]
        return _lib.FFBP_FINAL_TC_F16 | flags
    choice = os.environ.get('FASTSAR_FINAL', 'fp32').strip().lower() or 'fp32'
    if choice not in ('fp32', 'tc3'):
        raise ValueError(f"FASTSAR_FINAL must be 'fp32' or 'tc3', got {choice!r}")
    return _lib.FFBP_FINAL_TC_BF16X3 if choice == 'tc3' else _lib.FFBP_FINAL_FP32


class DevicePlan:
    """A plan of fastsar_b200.plan uploaded through ffbp_plan_create: the device-resident filters, windows, child
    phases and final-stage geometry, and the workspace of a form call. Owns the library's plan handle."""

    def __init__(self, plan, wp=None, wk=None, wf=None, ref=None, final_mode=_lib.FFBP_FINAL_FP32, device=None,
                 partial=False):
        import torch
        L = _lib.load()
        self.plan = plan
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        keep = []                                   # host arrays the descriptors point to, alive until the call returns

        def k64(a):
            a = _lib.c64(a)
            keep.append(a)
            return a.ctypes.data

        def k32(a):
            a = _lib.c32(a)
            keep.append(a)
            return a.ctypes.data

        lvs = (_lib.LevelDesc * len(plan['levels']))()
        for i, lv in enumerate(plan['levels']):
            d = lvs[i]
            d.sx, d.sy, d.C, d.Dk, d.Dp = lv['sx'], lv['sy'], lv['C'], lv['Dk'], lv['Dp']
            d.K, d.P, d.Ko, d.Po = lv['K'], lv['P'], lv['Ko'], lv['Po']
            if lv['fir_k'] is not None:
                d.h_taps_k, d.Lk, d.plk = k32(lv['fir_k']['kern']), lv['fir_k']['L'], lv['fir_k']['pl']
            if lv['fir_p'] is not None:
                d.h_taps_p, d.Lp, d.plp = k32(lv['fir_p']['kern']), lv['fir_p']['L'], lv['fir_p']['pl']
            d.f0, d.df = lv['f0'], lv['df']
            d.h_ant, d.h_ref, d.h_cen = k64(lv['ant']), k64(lv['ref']), k64(lv['cen'])
            if i == 0 and ref is not None:
                d.h_range = k64(ref)
            tc = lv.get('tc') or {}
            d.tc.nt, d.tc.sb, d.tc.copies, d.tc.repeat, d.tc.fir, d.tc.consumers = (
                int(tc.get(k, 0)) for k in ('nt', 'sb', 'copies', 'repeat', 'fir', 'consumers'))
        fin = plan['final']
        pd = _lib.PlanDesc()
        pd.nlev, pd.levels = len(plan['levels']), ctypes.cast(lvs, ctypes.POINTER(_lib.LevelDesc))
        pd.T, pd.nx, pd.ny, pd.Nx, pd.Ny, pd.ox, pd.oy = plan['T'], plan['nx'], plan['ny'], plan['Nx'], plan['Ny'], plan['ox'], plan['oy']
        pd.spx, pd.spy = plan['spx'], plan['spy']
        pd.e1[:] = list(map(float, plan['e1']))
        pd.e2[:] = list(map(float, plan['e2']))
        pd.Pf, pd.Qf, pd.f0f, pd.dff, pd.fcf = fin['P'], fin['K'], fin['f0'], fin['df'], fin['fc']
        pd.h_ant_f, pd.h_cen_f = k64(fin['ant']), k64(fin['cen'])
        first = np.ascontiguousarray(fin['first'], np.int32)
        keep.append(first)
        pd.h_first_f = first.ctypes.data
        if wp is not None:
            pd.h_wp, pd.h_wk = k32(wp), k32(wk)
        if wf is not None:
            pd.h_wf, pd.wf_ndim = k32(wf), int(wf.ndim)
        pd.final_mode = final_mode
        pd.partial = 1 if partial or plan.get('partial') else 0
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device)
            _lib.check(L.ffbp_plan_create(ctypes.byref(pd), ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)),
                       'ffbp_plan_create')
        del keep
        self.handle = h
        n = ctypes.c_size_t()
        _lib.check(L.ffbp_plan_workspace_bytes(h, ctypes.byref(n)), 'ffbp_plan_workspace_bytes')
        self.ws_bytes = int(n.value)
        self._ws = None
        self._stage = None

    def workspace(self):
        import torch
        if self._ws is None:
            try:
                self._ws = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=self.device)
            except torch.OutOfMemoryError:
                free, total = torch.cuda.mem_get_info(self.device)
                lv = self.plan['levels']
                raise MemoryError(
                    f'the plan needs {self.ws_bytes / 2**30:.1f} GiB of device workspace (the levels\' outputs and '
                    f'the tensor-core levels\' float16 intermediate) and {free / 2**30:.1f} of {total / 2**30:.1f} GiB '
                    f'are free on {self.device}; first-level children {lv[0]["C"]}, output samples per level '
                    f'{[l["Ko"] for l in lv]}, pulses {[l["Po"] for l in lv]}. Remedies: a smaller pmax (less '
                    'oversampling per level) or more levels, forming the image in parts (patches, or shard.ShardedFormer '
                    'over several GPUs), the range gate for an image narrow in range (range_gate=True), or freeing '
                    'other device memory') from None
        off = (-self._ws.data_ptr()) % 256
        return self._ws.data_ptr() + off

    def release_workspace(self):
        self._ws = None
        self._stage = None

    def form_host(self, S_ptrs, img_ptrs, stream=None):
        """ffbp_form_host on host buffers (addresses of [P, K] and [nx, ny] complex64 arrays, page-locked for the
        overlap): the images formed in turn, each upload and download overlapping the neighbours' formation.
        Returns each image's first non-finite pulse (-1: none)."""
        import torch
        L = _lib.load()
        n = len(S_ptrs)
        if self._stage is None:
            nb = ctypes.c_size_t()
            _lib.check(L.ffbp_plan_host_bytes(self.handle, ctypes.byref(nb)), 'ffbp_plan_host_bytes')
            self._stage_bytes = int(nb.value)
            self._stage = torch.empty(self._stage_bytes + 256, dtype=torch.uint8, device=self.device)
        stage = self._stage.data_ptr() + (-self._stage.data_ptr()) % 256
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        bad = (ctypes.c_int * n)()
        _lib.check(L.ffbp_form_host(self.handle, (ctypes.c_void_p * n)(*S_ptrs), (ctypes.c_void_p * n)(*img_ptrs), n,
                                    ctypes.c_void_p(stage), ctypes.c_size_t(self._stage_bytes),
                                    ctypes.c_void_p(self.workspace()), ctypes.c_size_t(self.ws_bytes),
                                    ctypes.c_void_p(stream.cuda_stream), bad), 'ffbp_form_host')
        return list(bad)

    def form(self, S_dev, img_dev, stream=None, check=True):
        """S_dev [P, K] complex64 torch tensor on the device -> img_dev [nx, ny] complex64 (written). check: read back
        the first non-finite pulse (a wait for the stream) and raise ValueError naming it, and RuntimeError when a
        tensor-core kernel of this call aborted. Without check nothing waits: an abort is raised by the next call
        or by check()."""
        import torch
        L = _lib.load()
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        bad = ctypes.c_int(-1)
        _lib.check(L.ffbp_form(self.handle, ctypes.c_void_p(S_dev.data_ptr()), ctypes.c_void_p(img_dev.data_ptr()),
                               ctypes.c_void_p(self.workspace()), ctypes.c_size_t(self.ws_bytes),
                               ctypes.c_void_p(stream.cuda_stream), ctypes.byref(bad) if check else None), 'ffbp_form')
        if check and bad.value >= 0:
            raise ValueError(f'phase history has non-finite samples (NaN or inf), the first in pulse {bad.value}; '
                             'zero them (S[~np.isfinite(S)] = 0) or drop the pulses')
        return img_dev

    def check(self, stream=None):
        """Wait for the stream and raise RuntimeError if a tensor-core kernel of an earlier form call (one made with
        check=False) aborted because a bounded wait of its pipeline ran out; its image is then incomplete. Each
        failure is raised once: here, or by the next form call."""
        import torch
        L = _lib.load()
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        _lib.check(L.ffbp_plan_check(self.handle, ctypes.c_void_p(stream.cuda_stream)), 'ffbp_plan_check')

    def test_wait(self, kind, limit_us=1000):
        """Test hook of the failure report: the MMA issuers of this plan's launches of `kind` ('level_tc' or
        'level_tc_gemm': the tensor-core levels in either form; 'final_tc'; None to turn it off) first wait limit_us microseconds on a barrier nothing completes, as a
        stuck pipeline's would, so that the kernel aborts and the failure is reported."""
        L = _lib.load()
        k = {None: 0, 'level_tc': _lib.FFBP_KIND_LEVEL_TC, 'level_tc_gemm': _lib.FFBP_KIND_LEVEL_TC_GEMM,
             'final_tc': _lib.FFBP_KIND_FINAL_TC}[kind]
        _lib.check(L.ffbp_plan_test_wait(self.handle, k, int(limit_us) if k else 0), 'ffbp_plan_test_wait')

    def test_transfer(self, image):
        """Test hook of the transfer check: the next form_many call leaves out the upload of its image `image` (the
        device buffer keeps what it held), as a transfer that did not deliver would; -1 turns it off."""
        _lib.check(_lib.load().ffbp_plan_test_transfer(self.handle, int(image)), 'ffbp_plan_test_transfer')

    def form_timed(self, S_dev, img_dev, stream=None):
        """form with the device time (ms) of each launch: [level 0, ..., level nlev-1, final] (waits for the stream)."""
        import torch
        L = _lib.load()
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        n = len(self.plan['levels']) + 1
        ms = (ctypes.c_float * n)()
        _lib.check(L.ffbp_form_timed(self.handle, ctypes.c_void_p(S_dev.data_ptr()), ctypes.c_void_p(img_dev.data_ptr()),
                                     ctypes.c_void_p(self.workspace()), ctypes.c_size_t(self.ws_bytes),
                                     ctypes.c_void_p(stream.cuda_stream), ms, n), 'ffbp_form_timed')
        return list(ms)

    def form_profile(self, S_dev, img_dev, stream=None):
        """form with the device time (ms) of every launch: [(kind name, level, ms), ...] in launch order."""
        import torch
        L = _lib.load()
        stream = torch.cuda.current_stream(self.device) if stream is None else stream
        n = self.launches()
        ms, kind = (ctypes.c_float * n)(), (ctypes.c_int * n)()
        _lib.check(L.ffbp_form_profile(self.handle, ctypes.c_void_p(S_dev.data_ptr()), ctypes.c_void_p(img_dev.data_ptr()),
                                       ctypes.c_void_p(self.workspace()), ctypes.c_size_t(self.ws_bytes),
                                       ctypes.c_void_p(stream.cuda_stream), ms, kind, n), 'ffbp_form_profile')
        return [(_lib.KIND_NAMES.get(k >> 8, '?'), k & 0xff, float(m)) for k, m in zip(kind, ms)]

    def launches(self):
        """Kernels one form call launches."""
        L = _lib.load()
        nl, nk = ctypes.c_int(), ctypes.c_int()
        _lib.check(L.ffbp_plan_info(self.handle, ctypes.byref(nl), ctypes.byref(nk)), 'ffbp_plan_info')
        return int(nk.value)

    def __del__(self):
        h = getattr(self, 'handle', None)
        if h is not None and h.value:
            try:
                _lib.load().ffbp_plan_destroy(h)
            except Exception:
                pass
            self.handle = None


class ImageFormer:
    """Factorized backprojection set up once for a collection geometry and output grid, then called on phase
    histories (fastsar/api.py:312-677): former = ImageFormer(ant, fmin, df, K, nx, ny, spx, spy, e1, e2);
    img = former(S). Building plans the tiles and filters and computes the float64 geometry on the device; each call
    performs only the image formation. aperture_weight(points [m, 3], pulses [n]) -> W [n, m] applies a per-pixel
    weight of pulses in the final stage (final_weights); ref [P] is the one-way range each pulse is referenced to
    when it is not |ant|. One former must not be called from two threads at once.

    precision='float32' runs the float32 kernels with the reference's filters (70 dB stop band); 'float16' is the
    mixed-precision form: the levels and the final stage on the tensor cores (split bfloat16 products, a float16
    intermediate, float16 final operands, float32 accumulation) with 80 dB filters, whose smaller error leaves room
    for the reduced-precision arithmetic. Unlike the reference's precision='float16' (float16 storage on its own
    plan), this changes the plan's filters: 80 dB instead of 70 dB (unless atten is given); T is chosen as for
    'float32' (choose_T: 32 where its predicted error meets target_db, else 16; the tensor-core final stage takes
    both). atten (an extension of this package) sets the filters' stop band in dB.
    taps (an extension too): 'kaiser' (default, the reference's Kaiser-sinc decimators), 'learned' (the packaged
    learned decimation taps, fastsar_b200.learned: 8-output-sample filters where the network covers a level's
    decimation and pass fraction, Kaiser-sinc ones elsewhere) or a LearnedTaps instance. tune_levels (an extension):
    with precision='float16', time the tensor-core levels' launch options (columns per tile, operand stages, plane
    copies, row repeat, consumer warps, the pulse FIR on the tensor or the CUDA cores) per level shape on the GPU when the former is
    built (fastsar_b200.tune.tune_levels; cached
    per shape in the process); the choice changes the image at the rounding level only (about 1e-5 relative: a
    float16 rounding of the intermediate flipped here and there)."""

    def __init__(self, ant, fmin, df, K, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), *, backend='auto',
                 precision='float32', window=True, T='auto', levels=None, pmax=0.4, target_db=-40.0, aperture_weight=None,
                 ref=None, range_gate='auto', padded=None, atten=None, taps='kaiser', tune_levels=False):
        self.ant = _check_positions(ant)
        self.P, self.K = self.ant.shape[0], int(K)
        if self.K < 2:
            raise ValueError(f'K must be at least 2 frequency samples, got {K}')
        if not (np.isfinite(fmin) and np.isfinite(df) and fmin > 0 and df > 0):
            raise ValueError(f'fmin and df must be positive frequencies in Hz, got {fmin!r} and {df!r}')
        nx, ny, e1, e2 = _check_grid(nx, ny, spx, spy, e1, e2)
        self.backend = _backend(backend)
        if precision not in ('float32', 'float16'):
            raise ValueError("cuda precision: 'float32' or 'float16'")
        self.precision = precision
        if atten is None:
            atten = 80.0 if precision == 'float16' else 70.0
        if not (np.isfinite(atten) and 20.0 <= float(atten) <= 200.0):
            raise ValueError(f'atten must be a stop-band attenuation in dB between 20 and 200, got {atten!r}')
        self.atten = float(atten)
        if isinstance(taps, str):
            if taps not in ('kaiser', 'learned'):
                raise ValueError(f"taps must be 'kaiser', 'learned' or a LearnedTaps, got {taps!r}")
            if taps == 'learned':
                from .learned import LearnedTaps
                taps = LearnedTaps.load()
            else:
                taps = None
        elif not hasattr(taps, 'decimator'):
            raise ValueError(f"taps must be 'kaiser', 'learned' or a LearnedTaps, got {taps!r}")
        self.taps = taps
        self.window = window
        self.nx, self.ny = nx, ny
        self.predicted_error_db = None
        fmax = float(fmin) + self.K * float(df)
        if T == 'auto':
            T, err = _plan.choose_T(self.ant, fmax, nx, ny, spx, spy, e1, e2, target_db)
            if err > target_db:
                warnings.warn(f'predicted error {err:.1f} dB at T={T} misses target {target_db:.1f} dB '
                              '(short range for this pixel size)')
            self.predicted_error_db = float(err)
        if T not in (16, 32):
            raise ValueError(f'the final stage supports T=16 or T=32, not {T}')
        self.T = T
        if ref is not None and np.shape(ref) != (self.P,):
            raise ValueError(f'ref must hold one range per pulse ({self.P}), got shape {np.shape(ref)}')
        if ref is not None and not np.all(np.isfinite(ref)):
            raise ValueError('ref has non-finite values')
        if range_gate not in ('auto', True, False):
            raise ValueError(f"range_gate must be 'auto', True or False, got {range_gate!r}")
        if padded is not None and (aperture_weight is None or levels is None or len(padded[2]) != levels
                                   or not 0 <= padded[0] <= self.P - padded[1]):
            raise ValueError('padded=(first, count, pulse) goes with an aperture_weight, the levels of the plan that '
                             f'pulse is from and an aperture within the {self.P} pulses, got {padded!r}')
        def planned(col):
            nlev = 3 if levels is None else levels
            while True:
                try:
                    return _plan.make_plan(col, nx, ny, spx, spy, T=T, nlev=nlev, pmax=pmax, e1=e1, e2=e2,
                                           pulse=padded and padded[2], atten=self.atten, taps=self.taps), nlev
                except ValueError as e:
                    if levels is not None or 'cannot split' not in str(e) or nlev >= 8:
                        raise
                    nlev += 1

        col = Collect(fmin=float(fmin), df=float(df), K=self.K, ant=self.ant, res=0.5)
        plan, nlev = planned(col)
        # the range gate (fastsar/api.py:398-416): 'auto' where the first level's frequency filter would not fit the
        # level kernel (more than 256 taps: an image narrow in range from a wide-band collection), True wherever it
        # keeps fewer than half of the samples
        self.range_gate = None
        lk = plan['levels'][0]['fir_k']['L'] if plan['levels'][0]['fir_k'] else 1
        why = None
        if range_gate == 'auto' and aperture_weight is None and lk > 256:
            why = (f"the first level's frequency filter would have {lk} taps (range decimation "
                   f"{plan['levels'][0]['Dk']}), more than the level kernel holds (256)")
        if why or range_gate is True:
            g = _plan.gate_plan(self.ant, ref, float(fmin), float(df), self.K, nx, ny, spx, spy, e1, e2)
            kept = g['k1'] - g['k0']
            if g['N'] < g['Kp'] and kept < (self.K if why else self.K // 2):
                col = Collect(fmin=g['fmin'], df=g['df'], K=kept, ant=self.ant, res=0.5)
                plan, nlev = planned(col)
                self.range_gate = dict(g, K=self.K, kept=kept, note=(
                    f'range gate: each pulse cut to the {g["N"]} range bins about the image before formation, '
                    f'{kept} samples for {self.K}' + (f' ({why})' if why else '')))
                lk = plan['levels'][0]['fir_k']['L'] if plan['levels'][0]['fir_k'] else 1
        self.levels = nlev
        self._plan = plan
        if lk > 256:
            raise ValueError(f'the first level\'s frequency filter has {lk} taps (range decimation '
                             f"{plan['levels'][0]['Dk']}: an image narrow in range from a wide-band collection), more "
                             'than the level kernel holds (256); form with range_gate=True (or \'auto\', without an '
                             'aperture_weight), a wider image, or several')
        wf = None
        if aperture_weight is not None:
            wspan = dict(P=self.P) if padded is None else dict(P=int(padded[1]), first=int(padded[0]))
            wf = _plan.final_weights(plan, aperture_weight, grad=True, **wspan)
            G = plan['levels'][0]['C']
            w0 = wf[0].reshape(G, -1)
            big = np.abs(w0) > 1e-6 * np.maximum(np.abs(w0).max(1, keepdims=True), 1e-30)
            gyr = np.where(big, wf[2].reshape(G, -1) / np.where(w0 == 0, 1, w0), 0.0).astype(np.float32)
            wf = np.stack([wf[0], wf[1], gyr.reshape(wf[0].shape)]).astype(np.float32)
        wp = wk = None
        if window:
            self.wp, self.wk = wp, wk = _window(self.P, self.K)
        mode = _final_mode(precision)
        # the tensor-core levels' launch options, timed per level shape (fastsar_b200.tune.tune_levels; cached)
        self.level_opts = None
        if tune_levels and mode & _lib.FFBP_LEVELS_TC and mode & _lib.FFBP_LEVELS_TC2:
            from . import tune as _tune
            self.level_opts = _tune.tune_levels(plan)
        # a gated history is windowed in the gate, before its transforms; the former then takes it as it is
        self._dev = DevicePlan(plan, None if self.range_gate else wp, None if self.range_gate else wk, wf,
                               None if ref is None else np.asarray(ref, np.float64), mode)
        self._S = None
        self._img = None
        self._gate_dev = None

    # ------------------------------------------------------------------------------------------------ calls
    def memory(self):
        """What a call needs on the device and what is free: dict(backend, needed, available, full_speed, parts)."""
        import torch
        free, _ = torch.cuda.mem_get_info(self._dev.device)
        parts = dict(history=self.P * self.K * 8, workspace=self._dev.ws_bytes, image=self.nx * self.ny * 8)
        need = float(sum(parts.values()))
        return dict(backend=self.backend, needed=need, available=float(free), full_speed=need <= free, parts=parts)

    def stage(self, S):
        """The work of a call that precedes formation, done ahead of it; former(former.stage(S)) equals former(S).
        Here: S checked and uploaded to the device (a torch tensor)."""
        return self._upload(S)

    def _upload(self, S):
        import torch
        if isinstance(S, torch.Tensor):
            if tuple(S.shape) != (self.P, self.K):
                raise ValueError(f'phase history must be {(self.P, self.K)}, got {tuple(S.shape)}')
            if not S.is_complex():
                raise TypeError(f'phase history must be complex (complex64 or complex128), got {S.dtype}')
            return S.to(device=self._dev.device, dtype=torch.complex64).contiguous()
        S = _check_history(np.asarray(S), self.P)
        if S.shape != (self.P, self.K):
            raise ValueError(f'phase history must be {(self.P, self.K)}, got {S.shape}')
        S = np.ascontiguousarray(S, np.complex64)
        if self._S is None:
            self._S = torch.empty((self.P, self.K), dtype=torch.complex64, device=self._dev.device)
        self._S.copy_(torch.from_numpy(S), non_blocking=False)
        return self._S

    def release(self):
        """Return the former's device buffers (workspace, staging, gate) to the allocator; the next call makes
        them again."""
        self._dev.release_workspace()
        self._S = None
        self._gate_dev = None

    def _gate(self, S_dev):
        """The range gate on the device (fastsar/api.py:525-564, fastsar/ffbp_cuda.py:767-864): S_dev [P, K]
        complex64 -> the gated history [P, kept] complex64 (a buffer of the former), windowed; in blocks of pulses
        whose padded rows stay within 256 MB; the transforms by cuFFT. Raises ValueError naming the first pulse with
        a non-finite sample."""
        import torch
        L = _lib.load()
        g = self.range_gate
        dev = self._dev.device
        P, K, kept = self.P, self.K, g['kept']
        npl, Kp, N, k0, k1 = g['npl'], g['Kp'], g['N'], g['k0'], g['k1']
        if self._gate_dev is None:
            win = self.window
            self._gate_dev = dict(
                taper=torch.from_numpy(np.ascontiguousarray(g['taper'], np.float32)).to(dev),
                wp=torch.from_numpy(np.ascontiguousarray(self.wp, np.float32)).to(dev) if win else None,
                wk=torch.from_numpy(np.ascontiguousarray(self.wk, np.float32)).to(dev) if win else None,
                out=torch.empty((P, kept), dtype=torch.complex64, device=dev),
                bad=torch.empty(1, dtype=torch.int32, device=dev))
        gd = self._gate_dev
        S_dev = S_dev.contiguous()
        gd['bad'].fill_(2 ** 31 - 1)
        stream = torch.cuda.current_stream(dev).cuda_stream
        nb = int(max(1, min(P, (1 << 28) // (Kp * 8))))
        tp = _lib.tptr
        for p0 in range(0, P, nb):
            r = min(nb, P - p0)
            z = torch.empty((r, Kp), dtype=torch.complex64, device=dev)
            _lib.check(L.ffbp_gate_pad(S_dev.data_ptr() + p0 * K * 8, r, K, tp(gd['wp']), tp(gd['wk']), npl, Kp,
                                       z.data_ptr(), gd['bad'].data_ptr(), p0, stream), 'ffbp_gate_pad')
            q = torch.fft.ifft(z, dim=1)
            del z
            u = torch.empty((r, N), dtype=torch.complex64, device=dev)
            _lib.check(L.ffbp_gate_fold(q.data_ptr(), r, Kp, N, u.data_ptr(), stream), 'ffbp_gate_fold')
            del q
            v = torch.fft.fft(u, dim=1)
            _lib.check(L.ffbp_gate_taper(v.data_ptr(), r, N, k0, k1, gd['taper'].data_ptr(),
                                         gd['out'].data_ptr() + p0 * kept * 8, stream), 'ffbp_gate_taper')
        b = int(gd['bad'].item())
        if b != 2 ** 31 - 1:
            raise ValueError(f'phase history has non-finite samples (NaN or inf), the first in pulse {b}; '
                             'zero them (S[~np.isfinite(S)] = 0) or drop the pulses')
        return gd['out']

    def form_device(self, S_dev, out=None, check=True):
        """S_dev [P, K] complex64 on the device -> the image [nx, ny] complex64 on the device (torch). With a range
        gate the history is gated first (and always checked for non-finite samples there)."""
        import torch
        if out is None:
            out = torch.empty((self.nx, self.ny), dtype=torch.complex64, device=self._dev.device)
        if self.range_gate is not None:
            if tuple(S_dev.shape) != (self.P, self.K):
                raise ValueError(f'phase history must be {(self.P, self.K)}, got {tuple(S_dev.shape)}')
            S_dev = self._gate(S_dev)
        return self._dev.form(S_dev, out, check=check)

    def check(self):
        """Wait for the device and raise RuntimeError if a tensor-core kernel of an earlier form_device(check=False)
        call aborted (a bounded wait of its pipeline ran out, leaving that image incomplete); the next form call
        raises it otherwise. Each failure is raised once."""
        self._dev.check()

    def form_many(self, histories, images=None):
        """Form a sequence of images from host memory: histories [P, K] complex64 (torch CPU tensors or numpy
        arrays; page-locked torch tensors, `pin_memory=True`, let the copies overlap the formation) -> images
        [nx, ny] complex64 in host memory (the given `images`, or new page-locked tensors), returned as numpy
        arrays. Each history's upload and each image's download run on their own streams while the neighbouring
        images form (ffbp_form_host). Every upload is checked by a sampled checksum on both sides of the transfer
        (the reference's transfer check): RuntimeError naming the first history that did not arrive as it is in host
        memory. Raises ValueError naming the first image with non-finite samples."""
        import torch
        hs = []
        for S in histories:
            if isinstance(S, torch.Tensor):
                if S.is_cuda:
                    raise ValueError('form_many takes host histories; use form_device for device ones')
                if tuple(S.shape) != (self.P, self.K) or S.dtype != torch.complex64 or not S.is_contiguous():
                    raise ValueError(f'host phase history must be a contiguous complex64 {(self.P, self.K)} tensor, '
                                     f'got {S.dtype} {tuple(S.shape)}')
                hs.append(S)
            else:
                S = _check_history(np.asarray(S), self.P)
                if S.shape != (self.P, self.K):
                    raise ValueError(f'phase history must be {(self.P, self.K)}, got {S.shape}')
                hs.append(torch.from_numpy(np.ascontiguousarray(S, np.complex64)))
        if images is None:
            images = [torch.empty((self.nx, self.ny), dtype=torch.complex64, pin_memory=True) for _ in hs]
        outs = []
        for im in images:
            t = im if isinstance(im, torch.Tensor) else torch.from_numpy(im)
            if tuple(t.shape) != (self.nx, self.ny) or t.dtype != torch.complex64 or not t.is_contiguous() or t.is_cuda:
                raise ValueError(f'images must be contiguous complex64 {(self.nx, self.ny)} host arrays')
            outs.append(t)
        if len(outs) != len(hs):
            raise ValueError(f'{len(hs)} histories but {len(outs)} images')
        if not hs:
            return []
        if self.range_gate is not None:                         # gated: one image after the other
            for i, (h, o) in enumerate(zip(hs, outs)):
                try:
                    o.copy_(self.form_device(h.to(self._dev.device)))
                except ValueError as e:
                    raise ValueError(str(e).replace('phase history', f'phase history {i}', 1)) from None
            return [o.numpy() for o in outs]
        bad = self._dev.form_host([h.data_ptr() for h in hs], [o.data_ptr() for o in outs])
        for i, b in enumerate(bad):
            if b >= 0:
                raise ValueError(f'phase history {i} has non-finite samples (NaN or inf), the first in pulse {b}; '
                                 'zero them (S[~np.isfinite(S)] = 0) or drop the pulses')
        return [o.numpy() for o in outs]

    def __call__(self, S):
        """S [P, K] complex phase history (numpy, or a torch tensor) -> complex64 image [nx, ny] (numpy)."""
        Sd = self._upload(S)
        img = self.form_device(Sd)
        return img.cpu().numpy()


class BatchFormer:
    """Several formers (patches of uneven sizes, from one or several collections; any precision and taps) formed
    together by one CUDA graph (ffbp_batch_create): each former's launches on a branch of their own, so that small
    images' kernels run side by side instead of one image after another, and one graph launch per batch. No
    counterpart in the reference, which forms a mosaic's patches one at a time (fastsar/patches.py:619-972).

    batch = BatchFormer([former_a, former_b, ...]); images = batch(histories) with host histories (numpy or torch
    CPU, each [P_i, K_i] complex) -> numpy images; or batch.form_device(device histories or None) -> the device
    images (None forms what batch.histories hold). sources[i]: the history former i forms from (formers of patches
    of one collection share it; default: a history per former); the histories passed are then one per source. The
    batch owns a device history per source and an image and a workspace per former (they run at once).
    Range-gated formers are not batched (the gate's transforms run outside the graph)."""

    def __init__(self, formers, sources=None):
        import torch
        L = _lib.load()
        self.formers = list(formers)
        if not self.formers:
            raise ValueError('BatchFormer needs at least one former')
        for i, f in enumerate(self.formers):
            if not isinstance(f, ImageFormer):
                raise TypeError(f'former {i} is not an ImageFormer')
            if f.range_gate is not None:
                raise ValueError(f'former {i} gates its history in range, which a batch does not run; '
                                 'form it alone')
        devs = {f._dev.device for f in self.formers}
        if len(devs) != 1:
            raise ValueError('the formers of a batch must be on one device')
        self.device = devs.pop()
        n = len(self.formers)
        self.sources = list(range(n)) if sources is None else [int(x) for x in sources]
        if len(self.sources) != n or min(self.sources) < 0:
            raise ValueError(f'sources must give each of the {n} formers a history index')
        shapes = {}
        for f, src in zip(self.formers, self.sources):
            if shapes.setdefault(src, (f.P, f.K)) != (f.P, f.K):
                raise ValueError(f'formers sharing history {src} differ in pulses or samples')
        if sorted(shapes) != list(range(len(shapes))):
            raise ValueError('sources must number the histories 0, 1, ... without gaps')
        self.histories = [torch.empty(shapes[k], dtype=torch.complex64, device=self.device) for k in range(len(shapes))]
        self.images = [torch.empty((f.nx, f.ny), dtype=torch.complex64, device=self.device) for f in self.formers]
        vp = ctypes.c_void_p
        plans = (vp * n)(*[f._dev.handle.value for f in self.formers])
        S = (vp * n)(*[self.histories[k].data_ptr() for k in self.sources])
        I = (vp * n)(*[m.data_ptr() for m in self.images])
        W = (vp * n)(*[f._dev.workspace() for f in self.formers])
        nb = (ctypes.c_size_t * n)(*[f._dev.ws_bytes for f in self.formers])
        h = vp()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device)
            _lib.check(L.ffbp_batch_create(plans, n, S, I, W, nb, vp(stream.cuda_stream), ctypes.byref(h)),
                       'ffbp_batch_create')
        self.handle = h

    def __del__(self):
        if getattr(self, 'handle', None) is not None and self.handle.value:
            try:
                _lib.load().ffbp_batch_destroy(self.handle)
            except Exception:
                pass
            self.handle = None

    def form_device(self, histories=None, check=True):
        """Device histories (torch tensors [P_i, K_i], complex) copied into the batch's buffers, or None for what
        they hold; one graph launch forms every image -> the batch's device images. check: wait and raise
        ValueError naming the first image with a non-finite sample."""
        import torch
        L = _lib.load()
        if histories is not None:
            if len(histories) != len(self.histories):
                raise ValueError(f'{len(self.histories)} histories expected, got {len(histories)}')
            for i, (S, buf) in enumerate(zip(histories, self.histories)):
                if tuple(S.shape) != tuple(buf.shape):
                    raise ValueError(f'phase history {i} must be {tuple(buf.shape)}, got {tuple(S.shape)}')
                buf.copy_(S, non_blocking=True)
        n = len(self.formers)
        stream = torch.cuda.current_stream(self.device)
        bad = (ctypes.c_int * n)() if check else None
        _lib.check(L.ffbp_batch_form(self.handle, ctypes.c_void_p(stream.cuda_stream), bad), 'ffbp_batch_form')
        if check:
            for i, b in enumerate(bad):
                if b >= 0:
                    raise ValueError(f'phase history {self.sources[i]} (image {i}) has non-finite samples (NaN or '
                                     f'inf), the first in pulse {b}; zero them (S[~np.isfinite(S)] = 0) or drop the '
                                     'pulses')
        return self.images

    def check(self):
        """Wait for the device and raise RuntimeError if a tensor-core kernel of an earlier form_device(check=False)
        launch aborted (a bounded wait ran out), naming the image."""
        for i, f in enumerate(self.formers):
            try:
                f.check()
            except RuntimeError as e:
                raise RuntimeError(f'image {i}: {e}') from None

    def __call__(self, histories):
        """Host histories (one per source) -> numpy images."""
        import torch
        ts = []
        for i, (S, buf) in enumerate(zip(histories, self.histories)):
            if not isinstance(S, torch.Tensor):
                S = _check_history(np.asarray(S), buf.shape[0])
                S = torch.from_numpy(np.ascontiguousarray(S, np.complex64))
            ts.append(S)
        if len(ts) != len(self.histories):
            raise ValueError(f'{len(self.histories)} histories expected, got {len(ts)}')
        imgs = self.form_device([t.to(self.device, torch.complex64) for t in ts])
        return [m.cpu().numpy() for m in imgs]


def form_image(S, ant, fmin, df, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), *, algorithm='ffbp',
               backend='auto', precision='float32', window=True, T='auto', levels=None, pmax=0.4, pfa_guard=300.0,
               pfa_support='union', target_db=-40.0, ref=None, interp=None, upsample=None, center=None,
               range_gate='auto'):
    """The complex image [nx, ny] (complex64) in one call (fastsar/api.py:680-716): algorithm='ffbp' builds an
    ImageFormer, 'bp' an ExactFormer; 'pfa' (polar format) is not part of this package."""
    if algorithm not in ('ffbp', 'pfa', 'bp'):
        raise ValueError("algorithm must be 'ffbp', 'pfa' or 'bp'")
    if algorithm != 'bp':
        for n, v in (('interp', interp), ('upsample', upsample), ('center', center)):
            if v is not None:
                raise ValueError(f"{n} applies to exact backprojection (algorithm='bp'), not to algorithm={algorithm!r}")
    if algorithm == 'pfa':
        raise ValueError("algorithm='pfa' (polar format) is not part of fastsar_b200; use 'ffbp' or 'bp'")
    S = _check_history(np.asarray(S), len(_check_positions(ant)))
    if algorithm == 'bp':
        from .exact import ExactFormer
        return ExactFormer(ant, fmin, df, S.shape[1], nx, ny, spx, spy, e1, e2, backend=backend, window=window,
                           interp='cubic' if interp is None else interp, upsample=upsample, ref=ref, center=center)(S)
    return ImageFormer(ant, fmin, df, S.shape[1], nx, ny, spx, spy, e1, e2, backend=backend, precision=precision,
                       window=window, T=T, levels=levels, pmax=pmax, target_db=target_db, ref=ref,
                       range_gate=range_gate)(S)
