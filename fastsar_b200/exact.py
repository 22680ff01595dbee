"""Exact backprojection (the oracle family of the former): ExactFormer and backproject on the GPU, and the grid points
of form_image."""
import numpy as np

C = 299792458.0


def plane_points(nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), height=None):
    """Points [nx, ny, 3] of the form_image grid: pixel (i, j) at (i - nx/2) spx e1 + (j - ny/2) spy e2, optionally
    displaced along the plane normal (pointing up) by height [nx, ny] (fastsar/bp.py:351-361)."""
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    X, Y = np.meshgrid((np.arange(nx) - nx / 2.0) * spx, (np.arange(ny) - ny / 2.0) * spy, indexing='ij')
    p = X[..., None] * e1 + Y[..., None] * e2
    if height is not None:
        n = np.cross(e1, e2)
        n = n / np.linalg.norm(n) * np.sign(n[2] if abs(n[2]) > 1e-12 else 1.0)
        p = p + np.asarray(height, np.float64)[..., None] * n
    return p


def _range_compress_device(S, nfft):
    """S [p, K] complex (torch, device) -> [p, nfft] complex128 range profiles (zero delay at nfft // 2, the carrier of
    sample K // 2 removed, the unnormalised inverse transform; fastsar/bp.py:55-63) by cuFFT."""
    import torch
    P, K = S.shape
    h = K // 2
    pad = torch.zeros((P, nfft), dtype=torch.complex128, device=S.device)
    pad[:, :K - h] = S[:, h:]
    pad[:, nfft - h:] = S[:, :h]
    return torch.fft.fftshift(torch.fft.ifft(pad, dim=1), dim=1) * nfft


def backproject_device(S, ant, fmin, df, points, *, rcv=None, ref=None, upsample=8, window=True, chunk=256):
    """Exact backprojection at points [..., 3] on the GPU in float64 throughout (profiles, geometry, interpolation,
    phase, accumulation) -> complex128 torch tensor [...] on the device. S: [P, K] complex, numpy or torch."""
    import torch
    from . import _lib
    L = _lib.load()
    dev = torch.device('cuda', torch.cuda.current_device())
    St = S if isinstance(S, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(S))
    St = St.to(dev)
    P, K = St.shape
    tx = np.ascontiguousarray(ant, np.float64)
    if ref is None:
        ref = np.linalg.norm(tx, axis=1) if rcv is None else 0.5 * (np.linalg.norm(tx, axis=1) + np.linalg.norm(rcv, axis=1))
    if window:
        from .api import _window
        wp, wk = _window(P, K)
        w = torch.from_numpy((wp[:, None] * wk[None, :]).astype(np.float32)).to(dev)
        St = St.to(torch.complex64) * w
    pts_np = np.asarray(points, np.float64)
    shape = pts_np.shape[:-1]
    pts = torch.from_numpy(np.ascontiguousarray(pts_np.reshape(-1, 3))).to(dev)
    out = torch.zeros(pts.shape[0], dtype=torch.complex128, device=dev)
    nfft = 1 << int(np.ceil(np.log2(upsample * K)))
    inv_dr = 2.0 * df * nfft / C
    kcyc = 2.0 * (fmin + (K // 2) * df) / C
    txd = torch.from_numpy(tx).to(dev)
    rcd = None if rcv is None else torch.from_numpy(np.ascontiguousarray(rcv, np.float64)).to(dev)
    refd = torch.from_numpy(np.ascontiguousarray(ref, np.float64)).to(dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    for p0 in range(0, P, chunk):
        p1 = min(P, p0 + chunk)
        prof = _range_compress_device(St[p0:p1], nfft).contiguous()
        _lib.check(L.ffbp_bp_points_f64(prof.data_ptr(), p1 - p0, nfft, txd[p0:p1].data_ptr(),
                                        None if rcd is None else rcd[p0:p1].data_ptr(), refd[p0:p1].data_ptr(),
                                        pts.data_ptr(), pts.shape[0], inv_dr, kcyc, out.data_ptr(), s),
                   'ffbp_bp_points_f64')
        del prof
    return out.reshape(shape)


def backproject(S, ant, fmin, df, points, *, rcv=None, ref=None, backend='auto', upsample=8, window=True, chunk=256):
    """Complex image at points [..., 3] (complex64, numpy) by exact backprojection (fastsar/bp.py:303-348): ant [P, 3]
    the antenna (monostatic) or transmitter when rcv [P, 3] is given; ref [P] the one-way (or mean) reference range
    per pulse. Runs on the GPU in float64 throughout (the reference's cpu backend is float64 with float32 profiles)."""
    from .api import _backend, _check_history, _check_positions
    _backend(backend)
    S = _check_history(np.asarray(S))
    P, K = S.shape
    tx = _check_positions(ant, 'antenna (transmitter) positions', P)
    rcv = None if rcv is None else _check_positions(rcv, 'receiver positions', P)
    points = np.asarray(points, np.float64)
    if points.ndim < 1 or points.shape[-1] != 3 or points.size == 0:
        raise ValueError(f'points must be [..., 3] with at least one point, got shape {points.shape}')
    if ref is not None:
        ref = np.asarray(ref, np.float64)
        if ref.shape != (P,):
            raise ValueError(f'ref must hold one range per pulse, shape ({P},), got {ref.shape}')
    return backproject_device(S, tx, fmin, df, points, rcv=rcv, ref=ref, upsample=upsample, window=window,
                              chunk=chunk).cpu().numpy().astype(np.complex64)


# ------------------------------------------------------------------------------------------------- ExactFormer
TILES = ((32, 32), (16, 16), (8, 16), (8, 8))     # tile sizes (pixels along e1, e2), largest first
PHASE_LIMIT = 3e-4                                 # rad: the largest predicted phase error of the range expansion


def _distance_to_rectangle(ant, x0, e1, e2, a0, a1, b0, b1):
    """Per pulse the distance from ant [P, 3] to the rectangle x0 + a e1 + b e2, a0 <= a <= a1, b0 <= b <= b1 (e1, e2
    orthonormal): the antenna projected onto the plane, its plane coordinates clamped into the rectangle (the
    distance is convex on the plane, so this is its minimum; fastsar/exact.py:389-396)."""
    v = ant - x0
    a = np.clip(v @ e1, a0, a1)
    b = np.clip(v @ e2, b0, b1)
    return np.linalg.norm(v - a[:, None] * e1 - b[:, None] * e2, axis=1)


class ExactFormer:
    """Exact backprojection onto the grid of form_image, set up once for a collection geometry
    (fastsar/exact.py:404-801): former(S) -> complex64 image [nx, ny]. ant [P, 3] antenna phase centres
    (monostatic), fmin, df, K the frequency samples, ref [P] the range each pulse is referenced to (default |ant|),
    center the point the grid is centred on (default the origin), interp 'cubic' (default) or 'linear', upsample the
    range oversampling (default 8), chunk the pulses range-compressed at a time.

    Set-up (host, float64): the tile (the largest of 32 x 32, 16 x 16, 8 x 16, 8 x 8 pixels whose predicted phase
    error from the third-order range expansion, 4 pi f_max / c h^4 / (2 r^3), stays below 3e-4 rad; former.tile,
    former.predicted_error_db), the tile centres, and per pulse the window of range bins the grid can reach (with a
    tile of margin). A call, per chunk of pulses: the windowed history zero-padded to nfft = 2^ceil(log2(upsample
    K)) samples, its inverse FFT (cuFFT), and the tiled backprojection (CUDA, fastsar_b200/csrc/exact_tiles.cu),
    which stages each tile's band of every profile by bulk copies (the reachable window blo / W below stays part of
    the set-up: it decides whether the grid fits the profiles without ambiguity). backend accepts the reference's values; only 'auto' and 'cuda' run. profiles
    is accepted for compatibility; the profiles stay float32. One former must not be called from two threads at
    once."""

    def __init__(self, ant, fmin, df, K, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), *, backend='auto',
                 window=True, interp='cubic', upsample=None, ref=None, center=None, chunk=1024, profiles='auto'):
        import warnings
        from .api import _backend, _check_positions, _check_grid, _window
        if interp not in ('cubic', 'linear'):
            raise ValueError(f"interp must be 'cubic' or 'linear', got {interp!r}")
        if profiles not in ('auto', 'float32', 'float16', 'float16-pair'):
            raise ValueError(f"profiles must be 'auto', 'float32', 'float16' or 'float16-pair', got {profiles!r}")
        if profiles == 'float16-pair' and interp != 'linear':
            raise ValueError("profiles='float16-pair' applies to interp='linear'")
        self.profiles = 'float32'
        self.ant = _check_positions(ant)
        self.P = len(self.ant)
        if isinstance(K, bool) or not float(K).is_integer() or int(K) < 2:
            raise ValueError(f'K (frequency samples per pulse) must be an integer of at least 2, got {K!r}')
        self.K = int(K)
        if not (np.isfinite(fmin) and np.isfinite(df) and df > 0):
            raise ValueError(f'fmin must be a finite frequency and df a positive frequency spacing in Hz, got {fmin} and {df}')
        fmin, df = float(fmin), float(df)
        nx, ny, e1, e2 = _check_grid(nx, ny, spx, spy, e1, e2)
        self.nx, self.ny, self.spx, self.spy = int(nx), int(ny), float(spx), float(spy)
        self.e1, self.e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
        if center is None:
            self.center = np.zeros(3)
        else:
            try:
                self.center = np.asarray(center, np.float64)
            except (TypeError, ValueError):
                raise ValueError(f'center must be a point (a finite 3-vector) in meters, got {center!r}') from None
            if self.center.shape != (3,) or not np.isfinite(self.center).all():
                raise ValueError(f'center must be a point (a finite 3-vector) in meters, got {center!r}')
        if ref is None:
            self.ref = np.linalg.norm(self.ant, axis=1)
        else:
            self.ref = np.asarray(ref, np.float64)
            if self.ref.shape != (self.P,):
                raise ValueError(f'ref must hold one range per pulse, shape ({self.P},), got {self.ref.shape}')
            if not np.isfinite(self.ref).all():
                raise ValueError('ref has non-finite values (NaN or inf), the first in pulse '
                                 f'{int(np.argmax(~np.isfinite(self.ref)))}')
        self.cubic = interp == 'cubic'
        self.upsample = 8 if upsample is None else int(upsample)
        if self.upsample < 1:
            raise ValueError(f'upsample must be a positive integer, got {upsample!r}')
        self.chunk = int(chunk)
        if self.chunk < 1:
            raise ValueError(f'chunk must be a positive integer, got {chunk!r}')
        self.backend = _backend(backend)
        self.fmin, self.df, self.window = fmin, df, window
        self.nfft = 1 << int(np.ceil(np.log2(self.upsample * self.K)))
        self.inv_dr = 2.0 * df * self.nfft / C
        self.kcyc = 2.0 * (fmin + (self.K // 2) * df) / C
        self.wp, self.wk = _window(self.P, self.K) if window else (np.ones(self.P, np.float32), np.ones(self.K, np.float32))
        # the tile: the largest whose predicted phase error stays below PHASE_LIMIT (fastsar/exact.py:512-540)
        x0 = self.center + (-nx / 2.0) * spx * self.e1 + (-ny / 2.0) * spy * self.e2          # pixel (0, 0)
        rmin = float(_distance_to_rectangle(self.ant, x0, self.e1, self.e2, 0.0, (nx - 1) * spx, 0.0,
                                            (ny - 1) * spy).min())
        kmax = 4 * np.pi * (fmin + (self.K - 1) * df) / C
        best = None
        for tx, ty in TILES:
            h = 0.5 * np.hypot((tx - 1) * spx, (ty - 1) * spy)
            r = rmin - h
            if r < 4 * h:
                continue
            err = h ** 4 / (2 * r ** 3)
            best = (tx, ty, err, kmax * err)
            if kmax * err <= PHASE_LIMIT:
                break
        if best is None:
            raise ValueError(f'the grid comes within {rmin:.1f} m of the antenna, too close for the tiled range expansion '
                             'of ExactFormer; use fastsar_b200.backproject on fastsar_b200.plane_points of the grid')
        self.tx, self.ty, expansion_m, phase = best
        self.tile = (self.tx, self.ty)
        self.predicted_error_db = float(20 * np.log10(max(phase, 1e-30)))
        if phase > PHASE_LIMIT:
            warnings.warn(f'ExactFormer: at {rmin:.0f} m from the antenna, even {self.tx} by {self.ty} pixel tiles leave a '
                          f'predicted phase error of {phase:.1e} rad ({self.predicted_error_db:.1f} dB) from the range '
                          'expansion; fastsar_b200.backproject on fastsar_b200.plane_points of the grid is exact at any '
                          'range', UserWarning, stacklevel=2)
        self.ntx, self.nty = -(-nx // self.tx), -(-ny // self.ty)
        bi = (np.arange(self.ntx) * self.tx + 0.5 * (self.tx - 1))[:, None, None]
        bj = (np.arange(self.nty) * self.ty + 0.5 * (self.ty - 1))[None, :, None]
        self.cen = np.ascontiguousarray((x0 + bi * spx * self.e1 + bj * spy * self.e2).reshape(-1, 3))
        # the bins each pulse can reach: the grid with a tile of margin, nearest by projection and clamping, farthest
        # at a corner, plus the expansion's error and the interpolation's taps (fastsar/exact.py:480-508)
        mx, my = self.tx * spx, self.ty * spy
        a0, a1, b0, b1 = -mx, (nx - 1) * spx + mx, -my, (ny - 1) * spy + my
        near = _distance_to_rectangle(self.ant, x0, self.e1, self.e2, a0, a1, b0, b1)
        corners = np.array([x0 + a * self.e1 + b * self.e2 for a in (a0, a1) for b in (b0, b1)])
        far = np.linalg.norm(corners[None] - self.ant[:, None], axis=2).max(1)
        slack = 4 + int(np.ceil(expansion_m * self.inv_dr))
        blo = np.floor((near - self.ref) * self.inv_dr).astype(np.int64) + self.nfft // 2 - slack
        bhi = np.ceil((far - self.ref) * self.inv_dr).astype(np.int64) + self.nfft // 2 + slack
        self.W = int((bhi - blo).max()) + 4
        near0 = _distance_to_rectangle(self.ant, x0, self.e1, self.e2, 0.0, (nx - 1) * spx, 0.0, (ny - 1) * spy)
        far0 = np.linalg.norm(np.array([x0 + a * self.e1 + b * self.e2 for a in (0.0, (nx - 1) * spx)
                                         for b in (0.0, (ny - 1) * spy)])[None] - self.ant[:, None], axis=2).max(1)
        need = int((np.ceil(far0 * self.inv_dr) - np.floor(near0 * self.inv_dr)).max()) + 2 * slack + 4
        if need > self.nfft:
            raise ValueError(f'the grid spans up to {float((far0 - near0).max()):.1f} m of range from one pulse, more than '
                             f'this collection resolves without ambiguity (c / (2 df) = {C / (2 * df):.1f} m less the '
                             f'interpolation margin: the grid needs {need} of the {self.nfft} range bins at '
                             f'upsample={self.upsample}); form a smaller grid (or several) or use samples spaced more '
                             'finely in frequency')
        self.blo = blo
        self.lo = (blo - self.nfft // 2).astype(np.int32)
        # consecutive blocks along the grid axis closer to constant range at mid-aperture (the less aligned with the
        # line of sight), so that resident blocks read the same bins from L2
        los = self.ant[self.P // 2] - self.center
        self.along1 = int(abs(los @ self.e1) <= abs(los @ self.e2))
        self._dev = None

    def memory(self):
        """What a call needs on the device: dict(backend, needed, available, full_speed, parts)."""
        import torch
        ch = min(self.chunk, self.P)
        parts = dict(history=self.P * self.K * 8, padded=ch * self.nfft * 8 * 2, image=self.nx * self.ny * 8)
        free, _ = torch.cuda.mem_get_info()
        need = float(sum(parts.values()))
        return dict(backend=self.backend, needed=need, available=float(free), full_speed=need <= free, parts=parts)

    def _upload(self):
        import torch
        if self._dev is None:
            dev = torch.device('cuda', torch.cuda.current_device())
            t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a if dt is None else a.astype(dt))).to(dev)
            self._dev = dict(ant=t(self.ant), ref=t(self.ref), cen=t(self.cen), wp=t(self.wp, np.float32),
                             wk=t(self.wk, np.float32))
        return self._dev

    def form_device(self, S_dev, check=True):
        """S_dev [P, K] complex64 torch tensor on the device -> complex64 image [nx, ny] on the device."""
        import ctypes
        import torch
        from . import _lib
        L = _lib.load()
        d = self._upload()
        dev = S_dev.device
        S_dev = S_dev.to(torch.complex64).contiguous()
        P, K, nfft = self.P, self.K, self.nfft
        ch = min(self.chunk, P)
        out = torch.zeros((self.nx, self.ny), dtype=torch.complex64, device=dev)
        pad = torch.zeros((ch, nfft), dtype=torch.complex64, device=dev)
        bad = torch.full((1,), 2 ** 31 - 1, dtype=torch.int32, device=dev)
        err = torch.zeros((1,), dtype=torch.int32, device=dev)
        s = torch.cuda.current_stream(dev).cuda_stream
        e1 = (ctypes.c_double * 3)(*self.e1)
        e2 = (ctypes.c_double * 3)(*self.e2)
        for p0 in range(0, P, ch):
            p1 = min(P, p0 + ch)
            n = p1 - p0
            _lib.check(L.ffbp_exact_pad(S_dev[p0:p1].data_ptr(), n, K, d['wp'].data_ptr(), d['wk'].data_ptr(), nfft,
                                        pad.data_ptr(), bad.data_ptr() if check else None, p0, s), 'ffbp_exact_pad')
            prof = torch.fft.ifft(pad[:n], dim=1)
            _lib.check(L.ffbp_exact_backproject(prof.data_ptr(), n, nfft, d['ant'][p0:p1].data_ptr(),
                                                d['ref'][p0:p1].data_ptr(), d['cen'].data_ptr(), self.ntx, self.nty,
                                                self.tx, self.ty, self.nx, self.ny, self.spx, self.spy, e1, e2,
                                                self.inv_dr, self.kcyc, int(self.cubic), self.along1, err.data_ptr(),
                                                out.data_ptr(), s), 'ffbp_exact_backproject')
            del prof
        if int(err.item()):
            raise RuntimeError('ffbp_exact_backproject: a bounded wait for the profiles ran out; the image is incomplete')
        if check:
            b = int(bad.item())
            if b != 2 ** 31 - 1:
                raise ValueError(f'phase history has non-finite samples (NaN or inf), the first in pulse {b}; '
                                 'zero them (S[~np.isfinite(S)] = 0) or drop the pulses')
        return out

    def __call__(self, S):
        """S [P, K] complex phase history (numpy, or a torch tensor) -> complex64 image [nx, ny] (numpy)."""
        import torch
        from .api import _check_history
        S = _check_history(S if isinstance(S, torch.Tensor) else np.asarray(S), self.P)
        if S.shape[1] != self.K:
            raise ValueError(f'phase history must have {self.K} samples per pulse, got {S.shape[1]}')
        if isinstance(S, np.ndarray):
            S = torch.from_numpy(np.ascontiguousarray(S.astype(np.complex64, copy=False)))
        return self.form_device(S.to(torch.device('cuda', torch.cuda.current_device()))).cpu().numpy()
