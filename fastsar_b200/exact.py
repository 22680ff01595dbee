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
