"""Pair products of images formed on one grid, on the B200: multilook, interferogram, coherence.

The reference's fastsar/products.py:28-67 (multilook, interferogram, coherence), with the same arguments and
results; each is one kernel of fastsar_b200/csrc/products.cu behind the C ABI (ffbp_multilook, ffbp_coherence).
Images are numpy arrays (the result comes back to the host) or torch tensors (the result stays on the device)."""
import ctypes

import numpy as np
import torch

from . import _lib


def device_image(x, dtype):
    """-> (a contiguous CUDA tensor of x as dtype, whether x came as a numpy array). Raises RuntimeError without a
    CUDA device: the products run only on the GPU."""
    if not torch.cuda.is_available():
        raise RuntimeError('fastsar_b200 stack products need a CUDA device (the kernels run on the GPU only)')
    host = not isinstance(x, torch.Tensor)
    t = torch.as_tensor(np.ascontiguousarray(x)) if host else x
    if t.ndim != 2:
        raise ValueError(f'an image is two-dimensional [n1, n2], got shape {tuple(t.shape)}')
    return t.to(device='cuda', dtype=dtype).contiguous(), host


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def give(t, host):
    return t.cpu().numpy() if host else t


def multilook(img, la=1, lr=1):
    """Power |img|^2 averaged over la x lr pixel boxes (axis 0, axis 1) and decimated by them: [n1 // la, n2 // lr]
    float32 (fastsar/products.py:28-32; the sums in float64)."""
    a, host = device_image(img, torch.complex64)
    la, lr = int(la), int(lr)
    out = torch.empty((a.shape[0] // max(la, 1), a.shape[1] // max(lr, 1)), dtype=torch.float32, device=a.device)
    _lib.check(_lib.load().ffbp_multilook(ptr(a), None, a.shape[0], a.shape[1], la, lr, ptr(out), stream_ptr()),
               'ffbp_multilook')
    return give(out, host)


def interferogram(a, b, la=1, lr=1):
    """Multilooked interferogram a conj(b) averaged over la x lr boxes and decimated, complex64
    (fastsar/products.py:42-50). a and b are formed on the same grid."""
    x, host = device_image(a, torch.complex64)
    y, _ = device_image(b, torch.complex64)
    if x.shape != y.shape:
        raise ValueError(f'the images of a pair share a grid: {tuple(x.shape)} and {tuple(y.shape)}')
    la, lr = int(la), int(lr)
    out = torch.empty((x.shape[0] // max(la, 1), x.shape[1] // max(lr, 1)), dtype=torch.complex64, device=x.device)
    _lib.check(_lib.load().ffbp_multilook(ptr(x), ptr(y), x.shape[0], x.shape[1], la, lr, ptr(out), stream_ptr()),
               'ffbp_multilook')
    return give(out, host)


def coherence(a, b, w1=5, w2=5):
    """Sample coherence |<a b*>| / sqrt(<|a|^2> <|b|^2>) over moving w1 x w2 windows, same shape as the images
    (fastsar/products.py:53-67: the windows of scipy.ndimage.uniform_filter with the edge pixels repeated), the sums
    in float64, the result float32. It is biased upward for few independent samples per window, as the reference
    states."""
    x, host = device_image(a, torch.complex64)
    y, _ = device_image(b, torch.complex64)
    if x.shape != y.shape:
        raise ValueError(f'the images of a pair share a grid: {tuple(x.shape)} and {tuple(y.shape)}')
    out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
    _lib.check(_lib.load().ffbp_coherence(ptr(x), ptr(y), x.shape[0], x.shape[1], int(w1), int(w2), ptr(out),
                                          stream_ptr()), 'ffbp_coherence')
    return give(out, host)
