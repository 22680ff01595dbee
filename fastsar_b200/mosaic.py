"""Long apertures and arbitrary tracks as patch mosaics on the B200 (fastsar/patches.py:156-972).

The scene's planar grid is cut into patches; each patch is formed by this package's ImageFormer from the pulses
that illuminate it, with the phase history re-referenced to the patch centre and gated in range to the patch, and
the patches are pasted into one image:

    from fastsar_b200 import mosaic
    img = mosaic.form_mosaic(fx, ant, origin, nx, ny, spx, spy, e1, e2, patch=(128, 128), crop=8,
                             beam=beam, awin='hann')

fx = dict(S [P, K], fmin, df, ref [P], band) is the FX phase history of the CPHD convention with per-pulse
reference ranges (a scatterer at x contributes exp(-4 pi i f_k (|x - a_p| - ref_p) / c)); pixel (i, j) of the grid
lies at origin + i spx e1 + j spy e2. Each patch (patch = (mx, my) pixels plus crop on each side) takes the pulses
for which beam(idx, points) -> u satisfies |u| <= umax at some of 9 x 9 points spread over it (all pulses without a
beam, or pulses=(lo, hi) / pulses(centre)), as one contiguous run; an azimuth window awin weighs pulse p at pixel x by
awin(u_p(x) / umax) in the former's final stage (ImageFormer's aperture_weight).

The per-patch history runs on the device (range_profiles, patch_history: cuFFT for the transforms, the kernels of
csrc/mosaic.cu for the padding with the re-referencing phase, the gate's gather and the gated spectrum's ramp and
taper). The reference's JAX and TPU program buckets (choose_buckets is kept, as a pure function) and its separable
weight terms (exact=True, FASTSAR_WEIGHT_TERMS=1) and stepped masks (amask=True) are not part of this module.
"""
import numpy as np

from . import _lib
from . import plan as _plan

C = 299792458.0
SUBS = ((1, 1), (1, 2), (2, 1), (2, 2), (2, 4), (4, 2), (4, 4))


# ------------------------------------------------------------------------------------------------ host helpers
def _taylor_fn(sll=35.0, nbar=4):
    """The Taylor window as a function of t in [-1, 1], 1 at t = 0: w(t) = 1 + 2 sum_m F_m cos(pi m t) with Taylor's
    coefficients F_m (m < nbar) for a peak side-lobe level of -sll dB (the published formula; stripmap.window's)."""
    A = np.arccosh(10.0 ** (float(sll) / 20.0)) / np.pi
    s2 = nbar ** 2 / (A ** 2 + (nbar - 0.5) ** 2)
    ms = np.arange(1, nbar)
    F = []
    for m in ms:
        num = np.prod([1.0 - m * m / s2 / (A ** 2 + (n - 0.5) ** 2) for n in ms])
        den = 2.0 * np.prod([1.0 - m * m / float(n * n) for n in ms if n != m])
        F.append((-1.0) ** (m + 1) * num / den)
    F = np.asarray(F)

    def w(t):
        t = np.asarray(t, np.float64)
        return 1.0 + 2.0 * np.tensordot(F, np.cos(np.pi * np.multiply.outer(ms, t)), axes=1)
    w0 = float(w(0.0))
    return lambda t: w(t) / w0


def window(spec):
    """An azimuth window as a function of t in [-1, 1], zero outside (fastsar/stripmap.py:158-176): None or 'none',
    'taylor' (35 dB, nbar 4), ('taylor', sll, nbar), 'hann', 'kaiser' (beta 2.5), ('kaiser', beta), or a callable."""
    if spec is None or (isinstance(spec, str) and spec == 'none'):
        fn = np.ones_like
    elif callable(spec):
        fn = spec
    else:
        name, *arg = (spec,) if isinstance(spec, str) else spec
        if name == 'taylor':
            fn = _taylor_fn(*arg)
        elif name == 'hann':
            fn = lambda t: 0.5 * (1.0 + np.cos(np.pi * np.clip(t, -1, 1)))
        elif name == 'kaiser':
            beta = float(arg[0]) if arg else 2.5
            fn = lambda t: np.i0(beta * np.sqrt(np.clip(1.0 - t * t, 0, 1))) / np.i0(beta)
        else:
            raise ValueError(f'unknown window {spec!r}')
    return lambda t: np.where(np.abs(t) <= 1, fn(np.clip(np.asarray(t, np.float64), -1, 1)), 0.0)


def _taper(f, band, guard):
    """1 over the band, a raised cosine to 0 across the guard on either side (fastsar/patches.py:156-159)."""
    t = np.clip(np.maximum(band[0] - f, f - band[1]) / guard, 0, 1)
    return 0.5 * (1.0 + np.cos(np.pi * t))


def _levels(n, T, most=3, longest=None):
    """The most levels (up to `most`) whose smallest split, 2 per level, does not pad n pixels beyond ceil(n / T)
    tiles; at least as many as split a longer side of `longest` pixels with factors of up to 16 per level
    (fastsar/patches.py:162-174)."""
    need = -(-n // T)
    nlev = max(1, min(most, int(np.floor(np.log2(max(need, 1))))))
    while longest is not None and nlev < most and 16 ** nlev < -(-longest // T):
        nlev += 1
    return nlev


def tile_plan(ant, fmax, px, py, spx, spy, e1, e2, target_db=-40.0, tiles=(32, 16), subs=SUBS):
    """The cheapest final tile size T and sub-grid factors (s1, s2) whose predicted final-stage error meets target_db
    (fastsar/patches.py:177-191): the patch is then formed at spacings spx / s1, spy / s2 and every s-th pixel kept.
    -> (T, (s1, s2), error dB); the smallest error found when none meets the target."""
    best = None
    for s1, s2 in subs:
        for T in tiles:
            err = _plan.final_phase_error(ant, fmax, px * s1, py * s2, spx / s1, spy / s2, e1, e2, T)
            if err <= target_db:
                return T, (s1, s2), float(err)
            if best is None or err < best[2]:
                best = (T, (s1, s2), float(err))
    return best


def beam_span(beam, P, pts, umax, step=64):
    """Pulses [lo, hi) for which |beam(p, x)| <= umax at some of the points pts, or None: the beam on every step-th
    pulse, then on every pulse only about the first and last found (a point's illuminated pulses are contiguous)
    (fastsar/patches.py:551-568)."""
    def lit(idx):
        return (np.abs(beam(idx, pts)) <= umax).any(1)
    coarse = np.unique(np.r_[np.arange(0, P, step), P - 1])
    hit = np.nonzero(lit(coarse))[0]
    if len(hit) == 0:
        every = np.nonzero(lit(np.arange(P)))[0]
        return None if len(every) == 0 else (int(every[0]), int(every[-1]) + 1)
    first = np.arange(int(coarse[hit[0] - 1]) if hit[0] > 0 else 0, int(coarse[hit[0]]) + 1)
    lo = int(first[np.nonzero(lit(first))[0][0]])
    end = int(coarse[hit[-1] + 1]) if hit[-1] + 1 < len(coarse) else P - 1
    last = np.arange(int(coarse[hit[-1]]), end + 1)
    hi = int(last[np.nonzero(lit(last))[0][-1]]) + 1
    return lo, hi


def fill_gaps(a):
    """Dropped pulses: where consecutive positions a [n, 3] lie m >= 2 median steps apart, m - 1 positions are
    inserted on the line between them (fastsar/patches.py:571-590). -> (positions [n', 3], index [n] of each original
    pulse among them); the inserted pulses carry zeros, which keep the pulse spacing even for the filters."""
    a = np.asarray(a, np.float64)
    step = np.linalg.norm(np.diff(a, axis=0), axis=1)
    med = float(np.median(step)) if len(step) else 0.0
    if not med > 0:
        return a, np.arange(len(a))
    m = np.maximum(np.rint(step / med).astype(np.int64), 1)
    if m.max() < 2:
        return a, np.arange(len(a))
    idx = np.concatenate([[0], np.cumsum(m)])
    out = np.empty((idx[-1] + 1, 3))
    for k in np.nonzero(m >= 2)[0]:
        f = np.arange(1, m[k])[:, None] / m[k]
        out[idx[k] + 1:idx[k + 1]] = (1 - f) * a[k] + f * a[k + 1]
    out[idx] = a
    return out, idx


def choose_buckets(counts, compile_cost, step=256):
    """Bucket pulse counts (multiples of step) for patches that share compiled programs (fastsar/patches.py:593-617):
    each patch takes the smallest bucket at least its count; minimizes compile_cost x buckets + the patches' padding
    work sum(bucket / count - 1), by dynamic programming over the distinct rounded counts. -> sorted bucket counts."""
    c = np.asarray(counts, np.int64).ravel()
    u, w = np.unique(step * -(-c[c > 0] // step), return_counts=True)
    if len(u) == 0:
        return []
    # padding of counts i..j up to u[j]: u[j] (A[j + 1] - A[i]) - (W[j + 1] - W[i]), prefix sums of w / u and of w
    A = np.concatenate([[0.0], np.cumsum(w / u)])
    W = np.concatenate([[0.0], np.cumsum(w.astype(np.float64))])
    best = np.zeros(len(u) + 1)
    back = np.empty(len(u), np.int64)
    for j in range(len(u)):
        cost = compile_cost + u[j] * (A[j + 1] - A[:j + 1]) - (W[j + 1] - W[:j + 1]) + best[:j + 1]
        i = int(np.argmin(cost))
        best[j + 1], back[j] = cost[i], i - 1
    out, j = [], len(u) - 1
    while j >= 0:
        out.append(int(u[j]))
        j = back[j]
    return out[::-1]


# ------------------------------------------------------------------------------------------------ patch histories
def _padding(fx, guard=None):
    """The frequency padding of fx to band +- guard (fastsar/patches.py:315-325): -> (guard, band, npl, K2, f0), K2
    a fast FFT length, f0 = fmin - npl df the padded axis's first frequency."""
    from scipy.fft import next_fast_len
    K = int(np.shape(fx['S'])[1])
    fmin, df = float(fx['fmin']), float(fx['df'])
    band = fx.get('band') or (fmin, fmin + (K - 1) * df)
    band = (float(band[0]), float(band[1]))
    room = min(band[0] - fmin, fmin + (K - 1) * df - band[1])
    guard = max(room, 0.125 * (band[1] - band[0])) if guard is None else float(guard)
    npl = max(0, int(np.ceil((fmin - band[0] + guard) / df)))
    npu = max(0, int(np.ceil((band[1] + guard - fmin - (K - 1) * df) / df)))
    return guard, band, npl, next_fast_len(K + npl + npu), fmin - npl * df


def _device_history(fx):
    """fx's history as a complex64 CUDA tensor (uploaded once and kept in fx under '_dev')."""
    import torch
    S = fx.get('_dev')
    if S is None:
        S = fx['S']
        S = S if isinstance(S, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(S))
        S = S.to(device='cuda', dtype=torch.complex64).contiguous()
    return S


def _stream():
    import ctypes
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def range_profiles(fx, guard=None):
    """The range profiles of the whole history, shared by a mosaic's patches (fastsar/patches.py:328-344): each pulse
    zero-padded to band +- guard and inverse-transformed, on the device. -> dict(Q [P, K2] complex64 tensor, guard,
    K2, npl, f0)."""
    import torch
    S = _device_history(fx)
    P, K = S.shape
    guard, band, npl, K2, f0 = _padding(fx, guard)
    Z = torch.empty((P, K2), dtype=torch.complex64, device=S.device)
    _lib.check(_lib.load().ffbp_mosaic_pad(S.data_ptr(), K, P, K, K2, npl, None, f0, float(fx['df']), Z.data_ptr(),
                                           _stream()), 'ffbp_mosaic_pad')
    return dict(Q=torch.fft.ifft(Z, dim=1), guard=guard, K2=K2, npl=npl, f0=f0)


def _gate_bins(a, rc, pts, margin, K2, df):
    """The range bins (of c / (2 K2 df)) a patch's gate keeps: the points' range extent from the antenna positions
    a [n, 3] (rc: their distances to the centre), from up to 513 of them, plus margin on each side; an even fast FFT
    length (fastsar/patches.py:347-356)."""
    from scipy.fft import next_fast_len
    k = np.unique(np.linspace(0, len(a) - 1, min(len(a), 513)).astype(np.int64))
    dR = np.linalg.norm(pts[None, :, :] - a[k, None, :], axis=2) - rc[k, None]
    half = np.abs(dR).max() + margin
    N = next_fast_len(2 * int(np.ceil(half * 2 * K2 * df / C)))
    return N + N % 2


def gate_bins(fx, ant, center, pts, lo, hi, margin=None, guard=None):
    """The range gate patch_history keeps for a patch, in bins: -> (N, K2) (fastsar/patches.py:359-364)."""
    guard, band, npl, K2, f0 = _padding(fx, guard)
    margin = 3 * C / (2 * guard) if margin is None else float(margin)
    a = np.asarray(ant[lo:hi], np.float64)
    return _gate_bins(a, np.linalg.norm(a - center, axis=1), pts, margin, K2, float(fx['df'])), K2


def _gate_samples(f0, df, K2, N, band, guard):
    """The samples of a history gated to N of its K2 range bins (all of them: no gate) (fastsar/patches.py:367-375):
    -> (gate, df', f' [N or K2], taper over them, k0, k1: the samples the taper does not zero)."""
    gate = N < K2
    df2 = K2 * df / N if gate else df
    f2 = f0 + df2 * np.arange(N if gate else K2)
    T = _taper(f2, band, guard)
    keep = np.nonzero(T > 0)[0]
    return gate, df2, f2, T, int(keep[0]), int(keep[-1]) + 1


def patch_history(fx, ant, center, pts, lo, hi, margin=None, guard=None, prof=None):
    """One patch's phase history (fastsar/patches.py:378-500): pulses lo:hi of fx re-referenced to center [3] (from
    ref_p to |a_p - center|) and gated in range to the extent of the points pts [m, 3] plus margin (m), with the guard
    taper; on the device. prof: range_profiles(fx, guard), shared by the patches: the gate is then gathered from the
    profiles (the whole-bin part of each pulse's delay an index offset, the fraction a phase ramp on the gated
    spectrum); without it the delay is a phase on the padded spectrum before the transforms.
    -> (S [hi - lo, K'] complex64 CUDA tensor, ant - center [hi - lo, 3], fmin', df')."""
    import torch
    L = _lib.load()
    S = _device_history(fx)
    df = float(fx['df'])
    K = S.shape[1]
    guard, band, npl, K2, f0 = _padding(fx, guard)
    margin = 3 * C / (2 * guard) if margin is None else float(margin)
    a = np.asarray(ant[lo:hi], np.float64)
    rows = hi - lo
    rc = np.linalg.norm(a - center, axis=1)
    shift = np.asarray(fx['ref'], np.float64)[lo:hi] - rc
    N = _gate_bins(a, rc, pts, margin, K2, df)
    gate, df2, f2, T, k0, k1 = _gate_samples(f0, df, K2, N, band, guard)
    dev = S.device
    taper = torch.as_tensor(T[k0:k1].astype(np.float32), device=dev)
    out = torch.empty((rows, k1 - k0), dtype=torch.complex64, device=dev)
    st = _stream()
    if gate and prof is not None:
        sft = 2 * df * K2 * shift / C
        m = np.rint(sft).astype(np.int64)
        Q = prof['Q'][lo:hi]
        u = torch.empty((rows, N), dtype=torch.complex64, device=dev)
        md = torch.as_tensor(m.astype(np.int32), device=dev)
        _lib.check(L.ffbp_mosaic_gather(Q.data_ptr(), K2, rows, K2, N, md.data_ptr(), u.data_ptr(), st),
                   'ffbp_mosaic_gather')
        U = torch.fft.fft(u, dim=1)
        del u
        d = torch.as_tensor(sft - m, device=dev)
        cph = torch.as_tensor(np.exp(-4j * np.pi * f0 * shift / C), device=dev)
        _lib.check(L.ffbp_mosaic_gate(U.data_ptr(), N, rows, k0, k1 - k0, N, d.data_ptr(), cph.data_ptr(), K2 / N,
                                      taper.data_ptr(), out.data_ptr(), st), 'ffbp_mosaic_gate')
        return out, a - center, float(f2[k0]), float(df2)
    sh = torch.as_tensor(shift, device=dev)
    S2 = torch.empty((rows, K2), dtype=torch.complex64, device=dev)
    _lib.check(L.ffbp_mosaic_pad(S[lo:hi].data_ptr(), K, rows, K, K2, npl, sh.data_ptr(), f0, df, S2.data_ptr(), st),
               'ffbp_mosaic_pad')
    if gate:
        q = torch.fft.ifft(S2, dim=1)
        del S2
        u = torch.empty((rows, N), dtype=torch.complex64, device=dev)
        _lib.check(L.ffbp_mosaic_gather(q.data_ptr(), K2, rows, K2, N, None, u.data_ptr(), st), 'ffbp_mosaic_gather')
        del q
        U = torch.fft.fft(u, dim=1)
        _lib.check(L.ffbp_mosaic_gate(U.data_ptr(), N, rows, k0, k1 - k0, N, None, None, K2 / N, taper.data_ptr(),
                                      out.data_ptr(), st), 'ffbp_mosaic_gate')
    else:
        _lib.check(L.ffbp_mosaic_gate(S2.data_ptr(), K2, rows, k0, k1 - k0, K2, None, None, 1.0, taper.data_ptr(),
                                      out.data_ptr(), st), 'ffbp_mosaic_gate')
    return out, a - center, float(f2[k0]), float(df2)


# ------------------------------------------------------------------------------------------------ the mosaic
def form_mosaic(fx, ant, origin, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), patch=(128, 128), crop=0,
                beam=None, umax=1.0, awin=None, pulses=None, margin=None, guard=None, backend='auto', T='auto',
                levels='auto', target_db=-40.0, sub='auto', info=None, precision='float32', exact=False, amask=False,
                device=False):
    """Complex image [nx, ny] (complex64) on the grid origin + i spx e1 + j spy e2 from the FX phase history fx
    (dict(S, fmin, df, ref[, band])) and the antenna positions ant [P, 3] of any track, formed patch by patch by
    this package's ImageFormer on the GPU (fastsar/patches.py:619-972, its cuda form).

    patch (mx, my) pixels per tile, each formed as a patch of (mx + 2 crop, my + 2 crop) pixels about the tile and
    cropped. beam(idx, points) -> u [len(idx), m]: a pulse serves a patch where |u| <= umax at one of 9 x 9 points of
    it; awin (a window spec, window()): pulse p weighted at pixel x by awin(u_p(x) / umax), clipped at the window's
    edges, in the former's final stage. pulses: (lo, hi) or a function of the patch centre, without a beam (default:
    all). margin, guard: the range gate's margin (m) and the spectral guard (Hz) (patch_history). T ('auto': 32 or
    16), sub ('auto' or (s1, s2)) and target_db choose each patch's final tile and sub-grid (tile_plan); levels
    ('auto': up to 3, _levels). precision: ImageFormer's. info: a list to which a dict per patch is appended
    (center, pulses, K, df, T, sub, levels, predicted error). device: return a torch CUDA tensor (else numpy).
    exact=True and amask=True (the reference's separable weight terms and stepped masks) are not part of this
    module."""
    import torch
    from .api import ImageFormer, _backend, _check_history, _check_positions, _check_grid
    _backend(backend)
    if exact or amask:
        raise ValueError('form_mosaic: exact=True and amask=True (separable weight terms, stepped masks) are not '
                         'part of fastsar_b200; the azimuth window is applied in the final stage')
    missing = [k for k in ('S', 'fmin', 'df', 'ref') if k not in fx]
    if missing:
        raise ValueError(f'fx lacks {missing}: a dict(S, fmin, df, ref[, band])')
    ant = _check_positions(ant)
    _check_history(fx['S'], len(ant))
    if np.shape(fx['ref']) != (len(ant),):
        raise ValueError(f"fx['ref'] must hold one reference range per pulse, shape ({len(ant)},), got "
                         f"{np.shape(fx['ref'])}")
    nx, ny, e1, e2 = _check_grid(nx, ny, spx, spy, e1, e2)
    if len(patch) != 2 or min(patch) < 1 or crop < 0:
        raise ValueError(f'patch must be two positive pixel counts and crop >= 0, got patch={patch!r}, crop={crop!r}')
    tiles = (32, 16) if T == 'auto' else (int(T),)
    subs = SUBS if sub == 'auto' else (tuple(sub),)
    o = np.asarray(origin, np.float64)
    e1v, e2v = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    mx, my = (int(v) for v in patch)
    px, py = mx + 2 * crop, my + 2 * crop
    wa = window(awin)
    wu = lambda u: wa(np.clip(u / umax, -1, 1))
    si, sj = np.linspace(0, px - 1, 9), np.linspace(0, py - 1, 9)
    gi, gj = np.meshgrid(si - px / 2, sj - py / 2, indexing='ij')
    fx = dict(fx)
    fx['_dev'] = _device_history(fx)
    out = torch.zeros((nx, ny), dtype=torch.complex64, device=fx['_dev'].device)
    npatch = -(-nx // mx) * -(-ny // my)
    # the shared range profiles [P, K2] where they take under 40 % of the free device memory (as the reference keeps
    # them on the device); else each patch transforms its own pulses (the direct form of patch_history)
    prof = None
    if npatch > 1:
        K2 = _padding(fx, guard)[3]
        free, _ = torch.cuda.mem_get_info(fx['_dev'].device)
        if 2 * len(ant) * K2 * 8 < 0.4 * free:          # the padded history and its transform
            prof = range_profiles(fx, guard)
    for i0 in range(0, nx, mx):
        for j0 in range(0, ny, my):
            c = o + (i0 - crop + px / 2) * spx * e1v + (j0 - crop + py / 2) * spy * e2v
            pts = c + (gi.ravel() * spx)[:, None] * e1v + (gj.ravel() * spy)[:, None] * e2v
            if beam is not None:
                span = beam_span(beam, len(ant), pts, umax)
            else:
                span = (0, len(ant)) if pulses is None else (pulses(c) if callable(pulses) else pulses)
            if span is None:
                continue
            lo, hi = (int(v) for v in span)
            Sp, a, f0, df2 = patch_history(fx, ant, c, pts, lo, hi, margin, guard, prof)
            Kp = int(Sp.shape[1])
            af, idx = fill_gaps(a)
            Tp, (s1, s2), err = tile_plan(af, f0 + Kp * df2, px, py, spx, spy, e1, e2, target_db, tiles, subs)
            nlev = (_levels(min(px * s1, py * s2), Tp, longest=max(px * s1, py * s2)) if levels == 'auto'
                    else int(levels))
            aw = None
            if beam is not None and awin is not None:
                def aw(q, pul, c=c, lo=lo, idx=idx):
                    # the window at points q (about the patch centre) for pulses pul of af (an inserted pulse takes
                    # the next recorded one's)
                    k = np.clip(np.searchsorted(idx, pul), 0, len(idx) - 1)
                    return wu(beam(lo + k, np.asarray(q) + c))
            former = ImageFormer(af, f0, df2, Kp, px * s1, py * s2, spx / s1, spy / s2, e1, e2,
                                 precision=precision, window=False, T=Tp, levels=nlev, aperture_weight=aw)
            if len(af) > len(idx):            # zero pulses at the inserted positions
                Z = torch.zeros((len(af), Kp), dtype=torch.complex64, device=Sp.device)
                Z[torch.as_tensor(idx, device=Sp.device)] = Sp
                Sp = Z
            img = former.form_device(Sp)[::s1, ::s2]
            ci, cj = min(mx, nx - i0), min(my, ny - j0)
            out[i0:i0 + ci, j0:j0 + cj] = img[crop:crop + ci, crop:crop + cj]
            former.release()
            del former, Sp, img
            if info is not None:
                info.append(dict(center=c, pulses=(lo, hi), K=Kp, df=df2, T=Tp, sub=(s1, s2), levels=nlev,
                                 predicted_error_db=err, terms=1))
    return out if device else out.cpu().numpy()
