"""Products of a repeat-pass stack on the B200: registration, translation and the incoherent average of images formed
on one grid.

The reference's fastsar/stack.py:485-1175, with its names, arguments and results:

  register(products, reference=0, apply=, max_shift=, tiles=, box=, highpass=)   fastsar/stack.py:929-1002
  shift_image(product, shift)                                                    fastsar/stack.py:770-831
  mean(products, equalize=, weights=, tile=)                                     fastsar/stack.py:1127-1190

and the steps they are made of (detected, peak, estimate, translate; the running average and its looks). The pixel
work runs in the kernels of fastsar_b200/csrc/products.cu (box means and decibels, the correlation's cross-spectrum
and energies, the ramp, the translation's crop, the average's sums and tile statistics), the transforms in cuFFT
(through torch.fft), the sub-pixel correlation's two small products in cuBLAS (complex128); the host handles only
per-image scalars and per-tile arrays.

A product is a dict with 'image' (complex or real, numpy or torch: a numpy image gives numpy results) and the grid's
'spx', 'spy' (m) and optionally 'origin', 'e1', 'e2' in the frame the image was formed in (ImageFormer's grid), as
the formers of this package produce them. The reference's products also carry their collection's frame (CPHD
metadata), from which it brings a complex image to baseband before translating it and re-forms on a displaced grid
(apply='reform') or refines on the complex images (coherent=True); those need the collection's geometry and are not
part of this module: a complex image is registered by estimate (apply=None), a real (detected) one also translated.
"""
import numpy as np
import torch
from scipy import fft as sfft

from . import _lib
from .products import device_image, give, ptr, stream_ptr


# ------------------------------------------------------------------------------------------------ pixel kernels
def intensity_box(x, w, to_db=False, kind=None):
    """The w x w box mean of the intensity of image x (CUDA tensor) in float32, or 10 log10 of it (to_db): the
    reference's _box(_power(x), w) bit for bit (fastsar/stack.py:485-528). kind: the pixel kind (default: the
    intensity of a complex image, the square of a real one); w = 1 gives the intensity itself."""
    if kind is None:
        kind = _lib.PIX_POWER if x.is_complex() else _lib.PIX_SQUARE
    out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
    _lib.check(_lib.load().ffbp_box_mean(ptr(x), int(kind), x.shape[0], x.shape[1], int(w), int(bool(to_db)), ptr(out),
                                         stream_ptr()), 'ffbp_box_mean')
    return out


def percentiles(v, qs):
    """Percentiles qs of a flat float32 CUDA tensor as numpy takes them of a float32 array: numpy's 'linear'
    method with the fraction q / 100, the virtual index (n - 1) q / 100 and the interpolation between the two order
    statistics about it all in float32 (so the same value to the bit). -> floats."""
    n = v.numel()
    if n == 0:
        raise ValueError('percentile of no pixels')
    s = torch.sort(v.reshape(-1).to(torch.float32)).values
    f32 = np.float32
    out = []
    for q in qs:
        h = f32(f32(n - 1) * f32(f32(q) / f32(100)))
        lo = int(np.floor(h))
        hi = min(lo + 1, n - 1)
        a, b = (f32(x) for x in s[[lo, hi]].cpu().numpy())
        t = f32(h - f32(lo))
        diff = f32(b - a)
        out.append(float(f32(a + f32(diff * t)) if t < 0.5 else f32(b - f32(diff * f32(1 - t)))))
    return out


def detected(img, box=5):
    """The image a registration correlates (fastsar/stack.py:543-549): the intensity averaged over box x box pixels,
    in decibels, clipped at its 1st and 99.5th percentiles (of every 4th pixel of every 4th row, the first and last
    sixteenth of the rows left out). Unprocessed pixels (0) take the lower clip. -> float32 CUDA tensor."""
    x, _ = device_image(img, _dtype_of(img))
    db = intensity_box(x, box, to_db=True)
    e = db.shape[0] // 16
    core = db[e:db.shape[0] - e] if e else db
    lo, hi = percentiles(core[::4, ::4].contiguous(), [1.0, 99.5])
    return torch.clamp(db, lo, float(np.float32(max(hi, lo + 1e-6))))


def _dtype_of(img):
    if isinstance(img, torch.Tensor):
        return torch.complex64 if img.is_complex() else torch.float32
    return torch.complex64 if np.iscomplexobj(img) else torch.float32


def _hann(n, device):
    return torch.as_tensor(np.hanning(n).astype(np.float32), device=device)


def _half_plane_weights(fs):
    m = np.arange(fs[1] // 2 + 1)
    return np.where((m == 0) | ((fs[1] % 2 == 0) & (m == fs[1] // 2)), 1.0, 2.0)


def peaks(a, b, max_shift, around=(0, 0), narrow=None, up=16, highpass=32.0):
    """peak of each pair of a batch: a, b [batch, n1, n2] float32 CUDA tensors, every pair searched about the same
    `around`. The pairs' transforms, cross-spectra, correlations and sub-pixel refinements each run as one batched
    call. -> a list of (d, z, rho, clear), one per pair."""
    nb, n1, n2 = a.shape
    dev = a.device
    h1, h2 = _hann(n1, dev), _hann(n2, dev)
    L = _lib.load()

    def windowed(x):      # ((x - its mean) w1) w2 per image, one pass (ffbp_window)
        x = x.contiguous()
        m = x.mean(dim=(1, 2)).contiguous()
        out = torch.empty_like(x)
        _lib.check(L.ffbp_window(ptr(x), nb, n1, n2, ptr(m), ptr(h1), ptr(h2), ptr(out), stream_ptr()), 'ffbp_window')
        return out
    aw, bw = windowed(a), windowed(b)
    fs = (sfft.next_fast_len(n1, real=True), sfft.next_fast_len(n2, real=True))
    A = torch.fft.rfft2(aw, s=fs).contiguous()
    B = torch.fft.rfft2(bw, s=fs).contiguous()
    m2h = fs[1] // 2 + 1
    X = torch.empty_like(A)
    energy = torch.empty((nb, 2), dtype=torch.float64, device=dev)
    e1 = e2 = None
    if highpass:
        s = 2.0 * np.pi * float(highpass) / 2.355
        k1, k2 = np.fft.fftfreq(fs[0]), np.fft.rfftfreq(fs[1])
        e1 = torch.as_tensor(np.exp(-0.5 * k1 * k1 * s * s).astype(np.float32), device=dev)
        e2 = torch.as_tensor(np.exp(-0.5 * k2 * k2 * s * s).astype(np.float32), device=dev)
    _lib.check(_lib.load().ffbp_cross_spectrum(ptr(A), ptr(B), nb, fs[0], m2h, int(fs[1] % 2 == 0), ptr(e1), ptr(e2),
                                               ptr(X), ptr(energy), stream_ptr()), 'ffbp_cross_spectrum')
    del A, B
    cc = torch.fft.irfft2(X, s=fs)
    m1_, m2_ = min(int(max_shift), fs[0] // 2 - 1), min(int(max_shift), fs[1] // 2 - 1)
    r1 = torch.as_tensor((int(around[0]) + np.arange(-m1_, m1_ + 1)) % fs[0], device=dev)
    r2 = torch.as_tensor((int(around[1]) + np.arange(-m2_, m2_ + 1)) % fs[1], device=dev)
    sub = cc.index_select(1, r1).index_select(2, r2).to(torch.float64)
    stats = torch.stack([cc.mean(dim=(1, 2)), cc.std(dim=(1, 2), unbiased=False)], 1).to(torch.float64)
    if highpass:
        norm = energy
    else:
        norm = torch.stack([(aw * aw).sum(dim=(1, 2)), (bw * bw).sum(dim=(1, 2))], 1).to(torch.float64)
    del cc, aw, bw
    sub, stats, norm = sub.cpu().numpy(), stats.cpu().numpy(), norm.cpu().numpy()
    out, fine_of = [], []
    for k in range(nb):
        i, j = np.unravel_index(int(np.argmax(sub[k])), sub[k].shape)
        top = sub[k][i, j]
        z = float((top - stats[k, 0]) / max(stats[k, 1], 1e-30))
        en = np.sqrt(norm[k, 0] * norm[k, 1])
        rho = float(top * fs[0] * fs[1] / max(en, 1e-30)) if highpass else float(top / max(en, 1e-30))
        d = np.array([i - m1_ + int(around[0]), j - m2_ + int(around[1])], np.float64)
        clear = 0 < i < 2 * m1_ and 0 < j < 2 * m2_
        if narrow is not None:
            clear = clear and abs(i - m1_) <= narrow and abs(j - m2_) <= narrow
        out.append([d, z, rho, bool(clear)])
        if clear and up > 1:
            fine_of.append(k)
    if not fine_of:
        return [tuple(o) for o in out]
    # the correlation about each clear peak at 1 / up of a pixel, from the half-plane spectrum, in float64 (the
    # complex64 spectrum widened through its float view, which is the fast path)
    t = np.arange(-up, up + 1) / up
    f64 = torch.float64
    f1 = torch.as_tensor(np.fft.fftfreq(fs[0]), device=dev)
    f2 = torch.as_tensor(np.fft.rfftfreq(fs[1]), device=dev)
    wk = torch.as_tensor(_half_plane_weights(fs), dtype=f64, device=dev)
    sel = torch.as_tensor(fine_of, device=dev)
    X2 = torch.view_as_complex(torch.view_as_real(X.index_select(0, sel)).to(f64))
    del X
    # the two factors of the upsampled inverse transform, exp(2 pi j (d + t) f), made on the device in float64
    d1 = torch.as_tensor(np.stack([out[k][0][0] + t for k in fine_of]), device=dev)          # [m, 2 up + 1]
    d2 = torch.as_tensor(np.stack([out[k][0][1] + t for k in fine_of]), device=dev)
    ph1 = (2 * np.pi) * d1[:, :, None] * f1[None, None, :]                                   # [m, 2 up + 1, fs0]
    ph2 = (2 * np.pi) * f2[None, :, None] * d2[:, None, :]                                   # [m, m2h, 2 up + 1]
    E1 = torch.polar(torch.ones_like(ph1), ph1)
    E2 = torch.polar(wk[None, :, None].expand_as(ph2).contiguous(), ph2)
    fine = torch.real(torch.bmm(torch.bmm(E1, X2), E2)).cpu().numpy()
    for q, k in enumerate(fine_of):
        fq = fine[q]
        i, j = np.unravel_index(int(np.argmax(fq)), fq.shape)
        off = np.array([t[i], t[j]])
        if 0 < i < 2 * up and 0 < j < 2 * up:
            off[0] += 0.5 * (fq[i - 1, j] - fq[i + 1, j]) / (fq[i - 1, j] - 2 * fq[i, j] + fq[i + 1, j]) / up
            off[1] += 0.5 * (fq[i, j - 1] - fq[i, j + 1]) / (fq[i, j - 1] - 2 * fq[i, j] + fq[i, j + 1]) / up
        out[k][0] = out[k][0] + off
        out[k][3] = True
    return [tuple(o) for o in out]


def peak(a, b, max_shift, around=(0, 0), narrow=None, up=16, highpass=32.0):
    """The translation d (pixels) at which b(x + d) best matches a(x), both float32 CUDA tensors (fastsar/stack.py:
    556-615): the maximum of their cross-correlation (means removed, Hann windows, the structure larger than
    `highpass` pixels removed by a Gaussian high pass) within max_shift of `around`, refined on the correlation
    upsampled `up` times about it and by a parabola. -> (d [2], z: the peak over the rms of the correlation surface,
    rho: the normalized correlation at the peak, clear: the peak off the search's border and, with narrow, within
    it of around)."""
    return peaks(a[None], b[None], max_shift, around, narrow, up, highpass)[0]


def estimate(ref, det, spx, spy, max_shift, tiles, highpass=32.0):
    """One translation between two detected images (CUDA tensors) and what tiles x tiles parts of them say after
    it (fastsar/stack.py:618-642): register's dict, shifts in pixels (shift_px) and meters (shift) along the grid
    axes. A peak counts as significant at 5 times the rms of its correlation surface. The parts are correlated as
    one batch."""
    d, z, rho, clear = peak(ref, det, max_shift, highpass=highpass)
    sp = np.array([spx, spy], np.float64)
    n1, n2 = ref.shape
    nt = int(tiles)
    T1, T2 = n1 // nt, n2 // nt
    res, zs, used = [], [], []
    ar = (int(round(d[0])), int(round(d[1])))
    if min(T1, T2) >= 48:
        def parts(x):     # [nt nt, T1, T2], the parts row by row
            return x[:nt * T1, :nt * T2].reshape(nt, T1, nt, T2).permute(0, 2, 1, 3).reshape(nt * nt, T1, T2)
        for dt, zt, _, ok in peaks(parts(ref), parts(det), max_shift, around=ar, narrow=8, highpass=highpass):
            res.append((dt - d) * sp)
            zs.append(zt)
            used.append(bool(ok and zt > 5.0))
    res, used = np.array(res).reshape(-1, 2), np.array(used, bool)
    rr = np.linalg.norm(res[used], axis=1) if used.any() else np.array([np.nan])
    return dict(shift_px=(float(d[0]), float(d[1])), shift=(float(d[0] * spx), float(d[1] * spy)), significance=z,
                correlation=rho, found=bool(clear and z > 5.0), tiles=nt * nt if len(res) else 0,
                tiles_used=int(used.sum()), tile_residuals=res, tile_used=used, tile_significance=np.array(zs),
                residual_rms=float(np.sqrt(np.mean(rr ** 2))), residual_median=float(np.median(rr)),
                residual_worst=float(rr.max()))


# ------------------------------------------------------------------------------------------------ translation
def translate(img, d):
    """img(x + d) for d = (d1, d2) pixels, img a CUDA tensor (fastsar/stack.py:685-725): the fraction of a pixel by a
    phase ramp exp(2 pi j k frac) on the spectrum of the image zero-padded by at least 16 samples along each axis
    (the whole sampled band; cuFFT), the whole pixels by moving the array (ffbp_shift_crop). Pixels whose source is
    outside the image, or exactly 0, are 0; a real image stays real (float32) and non-negative."""
    n1, n2 = img.shape
    d = np.asarray(d, np.float64)
    whole = np.rint(d).astype(int)
    frac = d - whole
    cplx = img.is_complex()
    src = img.to(torch.complex64 if cplx else torch.float32).contiguous()
    shifted, ld = None, n2
    if np.abs(frac).max() > 1e-6:
        fs = (sfft.next_fast_len(n1 + 16), sfft.next_fast_len(n2 + 16))
        F = torch.fft.fft2(src if cplx else src.to(torch.complex64), s=fs).contiguous()
        r1 = torch.as_tensor(np.exp(2j * np.pi * np.fft.fftfreq(fs[0]) * frac[0]).astype(np.complex64), device=src.device)
        r2 = torch.as_tensor(np.exp(2j * np.pi * np.fft.fftfreq(fs[1]) * frac[1]).astype(np.complex64), device=src.device)
        L = _lib.load()
        _lib.check(L.ffbp_ramp_multiply(ptr(F), fs[0], fs[1], ptr(r1), ptr(r2), stream_ptr()), 'ffbp_ramp_multiply')
        shifted = torch.fft.ifft2(F).contiguous()
        ld = fs[1]
        del F
    out = torch.empty_like(src)
    _lib.check(_lib.load().ffbp_shift_crop(ptr(shifted), ld, ptr(src), int(cplx), n1, n2, int(whole[0]), int(whole[1]),
                                           ptr(out), stream_ptr()), 'ffbp_shift_crop')
    return out


def _grid_of(p):
    """What names a product's pixels: shape, spacings and, when the product gives them, origin and axes."""
    img = p['image']
    g = dict(shape=tuple(int(v) for v in img.shape[:2]), spx=float(p['spx']), spy=float(p['spy']))
    for k in ('origin', 'e1', 'e2'):
        if p.get(k) is not None:
            g[k] = np.ravel(np.asarray(p[k], np.float64))
    return g


def _same_grid(a, b, tol=1e-3):
    """Whether two products' grids name the same pixels to tol of a pixel (fastsar/stack.py:189-195)."""
    if a['shape'] != b['shape'] or abs(a['spx'] - b['spx']) > 1e-9 or abs(a['spy'] - b['spy']) > 1e-9:
        return False
    n = max(a['shape'])
    for k, lim in (('origin', tol * min(a['spx'], a['spy'])), ('e1', tol / n), ('e2', tol / n)):
        if k in a and k in b and np.linalg.norm(a[k] - b[k]) >= lim:
            return False
    return True


def shift_image(out, shift):
    """A ground-plane product translated on its grid (fastsar/stack.py:770-831): pixel (i, j) of the result shows
    what the product has at (i, j) displaced by shift = (d1, d2) meters along e1 and e2. The whole pixels move the
    array, the fraction of a pixel is a phase ramp on the spectrum (translate); pixels shifted in from outside the
    image and pixels that were 0 are 0. shift (the product's entry) accumulates; origin, when the product gives it,
    moves with the translation. Real (detected) images only: a complex image is translated by the reference at
    baseband, from its collection's frame, which a product of this package does not carry."""
    if out.get('plane', 'ground') != 'ground':
        raise ValueError('shift_image takes a ground-plane product')
    img = out['image']
    if (img.is_complex() if isinstance(img, torch.Tensor) else np.iscomplexobj(img)):
        raise ValueError('shift_image: a complex image is translated at baseband from its collection frame, which '
                         'this product does not carry; translate its detected image, or register with apply=None')
    d1, d2 = (float(v) for v in shift)
    spx, spy = float(out['spx']), float(out['spy'])
    x, host = device_image(img, torch.float32)
    res = dict(out)
    res['image'] = give(translate(x, (d1 / spx, d2 / spy)), host)
    old = out.get('shift') or (0.0, 0.0)
    res['shift'] = (old[0] + d1, old[1] + d2)
    if out.get('origin') is not None and out.get('e1') is not None and out.get('e2') is not None:
        res['origin'] = (np.asarray(out['origin'], np.float64) + d1 * np.asarray(out['e1'], np.float64)
                         + d2 * np.asarray(out['e2'], np.float64))
    res['notes'] = list(out.get('notes', [])) + [
        f'translated by {d1:.3f} m along e1 and {d2:.3f} m along e2 on its grid (registration)']
    return res


def register(products, reference=0, *, apply='fourier', max_shift=64, tiles=4, box=5, highpass=32.0):
    """Register images formed on one grid: one translation each against a reference (fastsar/stack.py:929-1002).

    Each image gets the translation (d1, d2) at which it best matches the reference, image(x + d) ~ reference(x),
    from the peak of the cross-correlation of the detected images (detected: box x box mean intensity in dB,
    clipped), refined to a few hundredths of a pixel; its registration dict (estimate's) says how far to trust it
    (significance, found, and what tiles x tiles parts still disagree by after it). apply: 'fourier' translates the
    images whose peak was found (shift_image; real images: a complex product is estimated and left as it is, with
    a note), None estimates only. -> the list of products, each with 'registration' (the reference: shift (0, 0))."""
    if apply not in ('fourier', None, False):
        raise ValueError(f"apply must be 'fourier' or None, got {apply!r} (apply='reform' re-forms from the "
                         'collection, which the products of this package do not carry)')
    products = list(products)
    if not 0 <= reference < len(products):
        raise ValueError(f'reference {reference} is not one of the {len(products)} products')
    g0 = _grid_of(products[reference])
    for k, p in enumerate(products):
        if not _same_grid(g0, _grid_of(p)):
            raise ValueError(f'product {k} is not on the grid of the reference: form them on one grid')
    ref = detected(products[reference]['image'], box)
    out = []
    for k, p in enumerate(products):
        if k == reference:
            q = dict(p, registration=dict(shift=(0.0, 0.0), shift_px=(0.0, 0.0), reference=True))
            q.setdefault('shift', (0.0, 0.0))
            out.append(q)
            continue
        est = estimate(ref, detected(p['image'], box), float(p['spx']), float(p['spy']), max_shift, tiles, highpass)
        est['reference'] = False
        q = dict(p)
        img = p['image']
        cplx = img.is_complex() if isinstance(img, torch.Tensor) else np.iscomplexobj(img)
        if apply and est['found'] and not cplx:
            q = shift_image(p, est['shift'])
        elif apply:
            why = ('a complex image is not translated here (estimate only)' if est['found'] else
                   f"no significant correlation peak (significance {est['significance']:.1f})")
            q['notes'] = list(p.get('notes', [])) + [f'registration: {why}: not translated']
            q.setdefault('shift', (0.0, 0.0))
        q['registration'] = est
        out.append(q)
    return out


# ------------------------------------------------------------------------------------------------ the average
def _tiles_reduce(x, T, how):
    t1, t2 = x.shape[0] // T, x.shape[1] // T
    v = x[:t1 * T, :t2 * T].reshape(t1, T, t2, T)
    return (v.amax(dim=(1, 3)) if how == 'max' else v.amin(dim=(1, 3))).cpu().numpy()


def tile_stats(x, T, gain=1.0):
    """The mean and the (population) variance of x gain over each whole T x T tile of a float32 CUDA image:
    -> numpy [n1 // T, n2 // T] float32 each (fastsar/stack.py:1027-1034; float64 sums)."""
    t1, t2 = x.shape[0] // T, x.shape[1] // T
    m = torch.empty(max(t1 * t2, 1), dtype=torch.float32, device=x.device)
    v = torch.empty_like(m)
    _lib.check(_lib.load().ffbp_tile_stats(ptr(x), x.shape[0], x.shape[1], int(T), float(np.float32(gain)), ptr(m),
                                           ptr(v), stream_ptr()), 'ffbp_tile_stats')
    return m[:t1 * t2].reshape(t1, t2).cpu().numpy(), v[:t1 * t2].reshape(t1, t2).cpu().numpy()


def level(p, how):
    """An intensity image's brightness over its processed pixels, from every second pixel along both axes
    (fastsar/stack.py:1037-1048): the median, or the mean of the pixels up to their 99th percentile."""
    v = p[::2, ::2].reshape(-1)
    v = v[v > 0]
    n = v.numel()
    if n == 0:
        return 0.0
    if how == 'median':
        s = torch.sort(v).values
        mid = s[[(n - 1) // 2, n // 2]].cpu().numpy()
        return float(mid[0]) if n % 2 else float((mid[0] + mid[1]) / np.float32(2))
    t = percentiles(v, [99.0])[0]
    keep = v <= t
    r = torch.stack([torch.where(keep, v, torch.zeros((), dtype=v.dtype, device=v.device)).sum().to(torch.float64),
                     keep.sum().to(torch.float64)]).cpu().numpy()
    return float(np.float32(r[0])) / max(float(r[1]), 1.0)


class Mean:
    """The running incoherent average of images on one grid, on the device (fastsar/stack.py:1051-1124): each
    image's intensity times its weight (and, with equalize, the gain that brings its brightness to the first
    image's), summed per pixel with the sum of the weights of the images that processed it (ffbp_mean_add: the
    reference's float32 arithmetic, bit for bit); the tile statistics the looks are measured from."""

    def __init__(self, equalize, tile):
        self.equalize, self.T = equalize, int(tile)
        self.sum = self.wsum = self.first = None
        self.n, self.level0 = 0, None
        self.gains, self.single, self.running, self.inputs, self.weights = [], [], [], [], []
        self.host = False

    def add(self, out, weight=1.0):
        img = out['image']
        x, host = device_image(img, _dtype_of(img))
        kind = _lib.PIX_POWER if x.is_complex() else _lib.PIX_SQUARE
        p = intensity_box(x, 1, kind=kind)                    # the intensity itself
        g = 1.0
        if self.equalize:
            lv = level(p, self.equalize)
            if self.level0 is None:
                self.level0 = lv
            g = self.level0 / lv if lv > 0 else 1.0
        w = float(weight) * g
        first = self.sum is None
        if first:
            self.first, self.host = out, host
            self.sum = torch.empty(x.shape, dtype=torch.float32, device=x.device)
            self.wsum = torch.empty_like(self.sum)
        elif tuple(x.shape) != tuple(self.sum.shape):
            raise ValueError(f'image {self.n} is {tuple(x.shape)}, the first {tuple(self.sum.shape)}: the images of '
                             'a mean share a grid')
        _lib.check(_lib.load().ffbp_mean_add(ptr(x), kind, x.numel(), float(np.float32(w)), float(np.float32(weight)),
                                             int(first), ptr(self.sum), ptr(self.wsum), stream_ptr()), 'ffbp_mean_add')
        self.n += 1
        self.gains.append(g)
        self.weights.append(float(weight))
        if min(x.shape) >= 2 * self.T:
            self.single.append(tile_stats(p, self.T, np.float32(g)))
            self.running.append(tile_stats(self.image(), self.T))
        m = out.get('meta') or {}
        self.inputs.append(dict(name=m.get('core_name'), collector=m.get('collector'), start=str(m.get('start')),
                                shift=tuple(out.get('shift') or (0.0, 0.0)), gain=g, weight=float(weight),
                                graze=out.get('graze'), pulses=out.get('pulses'), band=out.get('band')))

    def image(self):
        M = torch.empty_like(self.sum)
        _lib.check(_lib.load().ffbp_mean_image(ptr(self.sum), ptr(self.wsum), self.sum.numel(), ptr(M), stream_ptr()),
                   'ffbp_mean_image')
        return M

    def looks(self, M):
        """The equivalent number of looks (mean^2 / variance of the intensity) on homogeneous tiles: of the tiles
        processed in every image, with a positive mean and no pixel above 6 times it, the 15 % whose 9 x 9 smoothed
        intensity varies least; the median over them (fastsar/stack.py:1096-1124)."""
        if not self.single:
            return dict(looks=None, tiles_selected=0)
        T = self.T
        mu, _ = tile_stats(M, T)
        top = _tiles_reduce(M, T, 'max')
        whole = _tiles_reduce(self.wsum, T, 'min') >= sum(self.weights) * (1 - 1e-6)
        sm_mean, sm_var = tile_stats(intensity_box(M, 9, kind=_lib.PIX_AS_IS), T)
        cv = np.sqrt(sm_var) / np.maximum(sm_mean, 1e-30)
        ok = (top < 6 * mu) & whole & (mu > 0)
        if ok.sum() < 8:
            return dict(looks=None, tiles_selected=0)
        hom = ok & (cv <= np.percentile(cv[ok], 15))

        def enl(s):
            return float(np.median(s[0][hom].astype(np.float64) ** 2 / np.maximum(s[1][hom].astype(np.float64), 1e-300)))
        single = [enl(s) for s in self.single]
        by_n = [enl(s) for s in self.running]
        mus = np.stack([s[0][hom] for s in self.single]).astype(np.float64)
        var = np.stack([s[1][hom] for s in self.single]).astype(np.float64)
        w = np.asarray(self.weights)[:, None]
        pred = float(np.median((w * mus).sum(0) ** 2 / np.maximum((w * w * var).sum(0), 1e-300)))
        spread = float(np.median(10 * np.log10(mus.max(0) / np.maximum(mus.min(0), 1e-300))))
        return dict(looks=by_n[-1], looks_single=single, looks_by_n=by_n, looks_ideal=self.n * float(np.mean(single)),
                    looks_independent=pred, brightness_spread_db=spread, tiles_selected=int(hom.sum()),
                    tiles=int(hom.size), tile=T, homogeneous=hom)


def mean(products, *, equalize=None, weights=None, tile=32):
    """The incoherent average of registered images of one scene: the mean of their intensities at full resolution
    (fastsar/stack.py:1127-1190), on the device.

    products: products on one grid, as a list or any iterable (a generator forms and gives up one image at a
    time). weights: one positive number per image (default equal). equalize: None, 'mean' or 'median': each image's
    intensity is first scaled by the factor that makes its brightness the first image's (the mean of the pixels under
    their 99th percentile, or the median, over the processed pixels). A pixel that is 0 in an image is left out of
    that pixel's average.

    -> a product with the first's other entries: image (the amplitude of the average, float32: its square is the
    mean intensity; on the device unless the first image came as a numpy array), product 'mean', count, looks (the
    equivalent number of looks of the average on homogeneous tiles; None for an image too small to measure),
    looks_single, looks_by_n, looks_ideal, looks_independent, brightness_spread_db, gains, inputs, tiles_selected,
    homogeneous, equalize."""
    if equalize not in (None, False, 'mean', 'median'):
        raise ValueError(f"equalize must be None, 'mean' or 'median', got {equalize!r}")
    acc = Mean(equalize or None, tile)
    g0 = None
    for k, p in enumerate(products):
        if p.get('plane', 'ground') != 'ground':
            raise ValueError('mean takes ground-plane products')
        g = _grid_of(p)
        if g0 is None:
            g0 = g
        elif not _same_grid(g0, g):
            raise ValueError(f'product {k} is not on the grid of the first: form them on one grid')
        w = 1.0 if weights is None else float(weights[k])
        if not w > 0:
            raise ValueError(f'weights must be positive, got {w!r}')
        acc.add(p, w)
    if acc.n == 0:
        raise ValueError('mean needs at least one product')
    M = acc.image()
    res = {k: v for k, v in acc.first.items() if k not in ('image', 'phase_error', 'registration', 'baseband', 'valid')}
    res.update(acc.looks(M))
    how = {None: 'as they are', 'mean': 'each scaled to the brightness of the first (mean under the 99th percentile)',
           'median': 'each scaled to the brightness of the first (median)'}[acc.equalize]
    res.update(image=give(torch.sqrt(M), acc.host), product='mean', count=acc.n, gains=list(acc.gains),
               inputs=acc.inputs, equalize=acc.equalize,
               notes=list(acc.first.get('notes', [])) + [f'incoherent average of {acc.n} images, {how}'])
    return res
