"""TEST INFRASTRUCTURE -- the oracle of the stack products. Only tests/ and bench.py's cpu_baseline / reference legs
import this module, to check the CUDA path (fastsar_b200.stack, fastsar_b200.products) or to time the CPU baseline.
The product never imports it.

A NumPy restatement, on the host cores, of what the reference computes after a stack of images is formed on a
common grid:

  registration   power, box, detected, peak, estimate      fastsar/stack.py:485-528, 535-549, 552-642
  translation    ramp, translate                           fastsar/stack.py:666-725 (the image's band: the whole
                                                           sampled band, as for a detected image)
  average        Mean (add, image, looks), level, tiles    fastsar/stack.py:1027-1124
  pair products  multilook, interferogram, coherence       fastsar/products.py:28-67

Parity is pinned: tests/test_stack_oracle.py checks every function here against the reference's own outputs on
seeded images (tests/golden/stack.npz, written by tests/golden/make_golden.py --only stack from saulpingerman/FastSAR
0.3.1): the float32 box sums bit for bit (the same additions in the same order), the rest to the rounding of the
transforms. Its transforms use every host core (scipy.fft workers=-1, as the reference's NumPy path does,
fastsar/stack.py:464-466).
"""
import numpy as np
from scipy import fft as sfft
from scipy.ndimage import uniform_filter


# ------------------------------------------------------------------------------------------------- registration
def power(img):
    """|img|^2 in float32 (fastsar/stack.py:485-490): re*re + im*im, each product rounded, for a complex image; the
    square of a real one."""
    img = np.asarray(img)
    if np.iscomplexobj(img):
        re, im = img.real.astype(np.float32), img.imag.astype(np.float32)
        return (re * re + im * im).astype(np.float32)
    x = img.astype(np.float32)
    return (x * x).astype(np.float32)


def box(x, w):
    """The mean over w x w pixels about each pixel, the edge pixels repeated (fastsar/stack.py:493-528): the window
    spans (w - 1) // 2 before and w // 2 after; the w rows are summed in order and divided by w, then the w columns
    likewise, in the array's own precision."""
    w = int(w)
    if w <= 1:
        return x
    before, after = (w - 1) // 2, w // 2
    out = x
    for axis in (0, 1):
        n = out.shape[axis]
        pad = [(0, 0), (0, 0)]
        pad[axis] = (before, after)
        ext = np.pad(out, pad, mode='edge')
        acc = np.take(ext, np.arange(0, n), axis=axis)
        for k in range(1, w):
            acc = acc + np.take(ext, np.arange(k, k + n), axis=axis)
        out = acc / w
    return out


def percentile(x, q, step=4):
    """Percentiles q (linear interpolation) of every step-th pixel along both axes (fastsar/stack.py:535-540)."""
    v = np.percentile(x[::step, ::step].ravel(), np.asarray(q, dtype=np.float32))
    return [float(t) for t in np.atleast_1d(v)]


def detected(img, w=5):
    """The image a registration correlates (fastsar/stack.py:543-549): the w x w mean of the intensity in dB, clipped
    at its 1st and 99.5th percentiles taken over all but the first and last sixteenth of the rows."""
    db = (10.0 * np.log10(np.maximum(box(power(img), w), 1e-30))).astype(np.float32)
    e = db.shape[0] // 16
    lo, hi = percentile(db[e:db.shape[0] - e] if e else db, [1.0, 99.5])
    return np.clip(db, lo, max(hi, lo + 1e-6)).astype(np.float32)


def hann(n):
    return np.hanning(n).astype(np.float32)


def highpass_filter(fs, cutoff):
    """The Gaussian high pass on the real transform's half plane (fastsar/stack.py:576-578): 1 - exp(-k^2 s^2 / 2)
    with s = 2 pi cutoff / 2.355 (cutoff: the structure size, pixels, at half power)."""
    k1, k2 = np.fft.fftfreq(fs[0])[:, None], np.fft.rfftfreq(fs[1])[None, :]
    s = 2.0 * np.pi * cutoff / 2.355
    return (1.0 - np.exp(-0.5 * (k1 * k1 + k2 * k2) * s * s)).astype(np.float32)


def half_plane_weights(fs):
    """The weight of each column of a real transform's half plane in a full-plane sum: 1 for the zero frequency
    and, for an even length, the Nyquist column; 2 for the others."""
    m = np.arange(fs[1] // 2 + 1)
    return np.where((m == 0) | ((fs[1] % 2 == 0) & (m == fs[1] // 2)), 1.0, 2.0)


def peak(a, b, max_shift, around=(0, 0), narrow=None, up=16, highpass=32.0):
    """The translation d at which b(x + d) best matches a(x) (fastsar/stack.py:556-615): the maximum of the
    cross-correlation of the two (means removed, Hann windows along both axes, high-passed) within max_shift of
    `around`, refined on the correlation upsampled `up` times about it and by a parabola through the samples
    about the finer maximum. -> (d [2], z: the peak over the rms of the correlation surface, rho: the normalized
    correlation at the peak, clear: the peak off the search's border (and within narrow of around))."""
    n1, n2 = a.shape
    win = hann(n1)[:, None] * hann(n2)[None, :]
    aw, bw = (a - a.mean()) * win, (b - b.mean()) * win
    fs = (sfft.next_fast_len(n1, real=True), sfft.next_fast_len(n2, real=True))
    A, B = sfft.rfft2(aw, s=fs, workers=-1), sfft.rfft2(bw, s=fs, workers=-1)
    X = np.conj(A) * B
    hp = None
    if highpass:
        hp = highpass_filter(fs, highpass)
        X = X * hp
    cc = sfft.irfft2(X, s=fs, workers=-1)
    m1, m2 = min(int(max_shift), fs[0] // 2 - 1), min(int(max_shift), fs[1] // 2 - 1)
    r1 = (int(around[0]) + np.arange(-m1, m1 + 1)) % fs[0]
    r2 = (int(around[1]) + np.arange(-m2, m2 + 1)) % fs[1]
    sub = cc[np.ix_(r1, r2)].astype(np.float64)
    i, j = np.unravel_index(int(np.argmax(sub)), sub.shape)
    top = sub[i, j]
    z = float((top - float(cc.mean())) / max(float(cc.std()), 1e-30))
    if hp is None:
        rho = float(top / max(np.sqrt(float((aw * aw).sum()) * float((bw * bw).sum())), 1e-30))
    else:
        wk = half_plane_weights(fs).astype(np.float32)[None, :] * hp
        ea, eb = float((np.abs(A) ** 2 * wk).sum()), float((np.abs(B) ** 2 * wk).sum())
        rho = float(top * fs[0] * fs[1] / max(np.sqrt(ea * eb), 1e-30))
    d = np.array([i - m1 + int(around[0]), j - m2 + int(around[1])], np.float64)
    clear = 0 < i < 2 * m1 and 0 < j < 2 * m2
    if narrow is not None:
        clear = clear and abs(i - m1) <= narrow and abs(j - m2) <= narrow
    if not clear or up <= 1:
        return d, z, rho, bool(clear)
    t = np.arange(-up, up + 1) / up
    E1 = np.exp(2j * np.pi * np.outer(d[0] + t, np.fft.fftfreq(fs[0])))
    E2 = np.exp(2j * np.pi * np.outer(np.fft.rfftfreq(fs[1]), d[1] + t)) * half_plane_weights(fs)[:, None]
    fine = np.real(E1 @ X.astype(np.complex128) @ E2)
    i, j = np.unravel_index(int(np.argmax(fine)), fine.shape)
    off = np.array([t[i], t[j]])
    if 0 < i < 2 * up and 0 < j < 2 * up:
        off[0] += 0.5 * (fine[i - 1, j] - fine[i + 1, j]) / (fine[i - 1, j] - 2 * fine[i, j] + fine[i + 1, j]) / up
        off[1] += 0.5 * (fine[i, j - 1] - fine[i, j + 1]) / (fine[i, j - 1] - 2 * fine[i, j] + fine[i, j + 1]) / up
    return d + off, z, rho, True


def estimate(ref, det, spx, spy, max_shift, tiles, highpass=32.0):
    """One translation between two detected images and what tiles x tiles parts of them say after it
    (fastsar/stack.py:618-642): each part's own peak searched within 8 pixels of the whole image's; a part counts
    when its peak is clear and its significance above 5."""
    d, z, rho, clear = peak(ref, det, max_shift, highpass=highpass)
    n1, n2 = ref.shape
    nt = int(tiles)
    T1, T2 = n1 // nt, n2 // nt
    res, zs, used = [], [], []
    ar = (int(round(d[0])), int(round(d[1])))
    if min(T1, T2) >= 48:
        for ti in range(nt):
            for tj in range(nt):
                sl = (slice(ti * T1, (ti + 1) * T1), slice(tj * T2, (tj + 1) * T2))
                dt, zt, _, ok = peak(ref[sl], det[sl], max_shift, around=ar, narrow=8, highpass=highpass)
                res.append((dt - d) * np.array([spx, spy]))
                zs.append(zt)
                used.append(bool(ok and zt > 5.0))
    res, used = np.array(res).reshape(-1, 2), np.array(used, bool)
    rr = np.linalg.norm(res[used], axis=1) if used.any() else np.array([np.nan])
    return dict(shift_px=(float(d[0]), float(d[1])), shift=(float(d[0] * spx), float(d[1] * spy)), significance=z,
                correlation=rho, found=bool(clear and z > 5.0), tiles=nt * nt if len(res) else 0,
                tiles_used=int(used.sum()), tile_residuals=res, tile_used=used, tile_significance=np.array(zs),
                residual_rms=float(np.sqrt(np.mean(rr ** 2))), residual_median=float(np.median(rr)),
                residual_worst=float(rr.max()))


# ------------------------------------------------------------------------------------------------- translation
def ramp(n, frac):
    """exp(2 pi j k frac) over the n samples' frequencies k (cycles per sample), complex64: the shift by frac of a
    sample of a signal occupying the whole sampled band (fastsar/stack.py:666-682 with the band limits at +-1/2,
    where the smooth step across an empty part of the band does not arise)."""
    return np.exp(2j * np.pi * np.fft.fftfreq(n) * frac).astype(np.complex64)


def translate(img, d):
    """img(x + d) for d = (d1, d2) pixels (fastsar/stack.py:685-725): the fraction by a phase ramp on the spectrum of
    the image zero-padded by at least 16 samples along each axis, the whole pixels by moving the array. Pixels whose
    source lies outside the image, and pixels that were exactly 0, are 0; a real image stays real and non-negative."""
    n1, n2 = img.shape
    d = np.asarray(d, np.float64)
    whole = np.rint(d).astype(int)
    frac = d - whole
    cplx = np.iscomplexobj(img)
    zero = img == 0
    out = img
    if np.abs(frac).max() > 1e-6:
        fs = (sfft.next_fast_len(n1 + 16), sfft.next_fast_len(n2 + 16))
        F = sfft.fft2(img if cplx else img.astype(np.complex64), s=fs, workers=-1)
        F = F * (ramp(fs[0], frac[0])[:, None] * ramp(fs[1], frac[1])[None, :])
        out = sfft.ifft2(F, workers=-1)[:n1, :n2]
        if not cplx:
            out = np.maximum(out.real, 0).astype(img.dtype)

    def moved(a, fill):
        if not whole.any():
            return a
        res = np.full(a.shape, fill, a.dtype)
        src = [slice(max(w, 0), min(n + w, n)) for n, w in zip(a.shape, whole)]
        if any(s.stop <= s.start for s in src):
            return res
        dst = tuple(slice(s.start - w, s.stop - w) for s, w in zip(src, whole))
        res[dst] = a[tuple(src)]
        return res
    out = moved(out, 0)
    if zero.any():
        out = np.where(moved(zero, True), np.zeros((), out.dtype), out)
    return out


# ------------------------------------------------------------------------------------------------- average
def tiles(x, T):
    """[n1 // T, n2 // T, T * T]: the whole T x T tiles of x, each flattened row by row."""
    n1, n2 = x.shape[0] // T, x.shape[1] // T
    return x[:n1 * T, :n2 * T].reshape(n1, T, n2, T).swapaxes(1, 2).reshape(n1, n2, T * T)


def tile_stats(x, T):
    t = tiles(x, T)
    return t.mean(-1), t.var(-1)


def level(p, how):
    """An intensity image's brightness over its processed pixels, from every second pixel along both axes
    (fastsar/stack.py:1037-1048): the median, or the mean of the pixels up to their 99th percentile."""
    v = p[::2, ::2].ravel()
    v = v[v > 0]
    if v.size == 0:
        return 0.0
    if how == 'median':
        return float(np.median(v))
    t = np.percentile(v, 99.0)
    keep = v <= t
    return float(np.where(keep, v, 0).sum() / max(int(keep.sum()), 1))


class Mean:
    """The running incoherent average of intensities on one grid (fastsar/stack.py:1051-1124): each image's
    intensity times its weight (and, with equalize, the gain that brings its level to the first image's), summed;
    a pixel's sum of weights counts the images in which it is processed (non-zero)."""

    def __init__(self, equalize=None, tile=32):
        self.equalize, self.T = equalize, int(tile)
        self.sum = self.wsum = None
        self.n, self.level0 = 0, None
        self.gains, self.weights, self.single, self.running = [], [], [], []

    def add(self, img, weight=1.0):
        p = power(img)
        g = 1.0
        if self.equalize:
            lv = level(p, self.equalize)
            if self.level0 is None:
                self.level0 = lv
            g = self.level0 / lv if lv > 0 else 1.0
        w = np.float32(float(weight) * g)
        valid = (p > 0).astype(np.float32) * np.float32(weight)
        if self.sum is None:
            self.sum, self.wsum = p * w, valid
        else:
            if p.shape != self.sum.shape:
                raise ValueError(f'image {self.n} is {p.shape}, the first {self.sum.shape}: the images share a grid')
            self.sum, self.wsum = self.sum + p * w, self.wsum + valid
        self.n += 1
        self.gains.append(g)
        self.weights.append(float(weight))
        if min(p.shape) >= 2 * self.T:
            self.single.append(tile_stats(p * np.float32(g), self.T))
            self.running.append(tile_stats(self.image(), self.T))

    def image(self):
        return np.where(self.wsum > 0, self.sum / np.maximum(self.wsum, 1e-30), 0).astype(np.float32)

    def looks(self, M):
        """The equivalent number of looks (mean^2 / variance) on homogeneous tiles: among the tiles processed in
        every image, with a positive mean and no pixel above 6 times it, the 15 % whose 9 x 9 smoothed intensity
        varies least (its coefficient of variation); the median over them."""
        if not self.single:
            return dict(looks=None, tiles_selected=0)
        T = self.T
        tm = tiles(M, T)
        mu = tm.mean(-1)
        whole = tiles(self.wsum, T).min(-1) >= sum(self.weights) * (1 - 1e-6)
        ts = tiles(box(M, 9), T)
        cv = ts.std(-1) / np.maximum(ts.mean(-1), 1e-30)
        ok = (tm.max(-1) < 6 * mu) & whole & (mu > 0)
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


# ------------------------------------------------------------------------------------------------- pair products
def multilook(img, la=1, lr=1):
    """|img|^2 averaged over la x lr boxes and decimated by them (fastsar/products.py:28-32)."""
    p = np.abs(np.asarray(img)) ** 2
    nx, ny = (p.shape[0] // la) * la, (p.shape[1] // lr) * lr
    return p[:nx, :ny].reshape(nx // la, la, ny // lr, lr).mean((1, 3))


def interferogram(a, b, la=1, lr=1):
    """a conj(b) averaged over la x lr boxes and decimated (fastsar/products.py:42-50)."""
    x = np.asarray(a) * np.conj(np.asarray(b))
    nx, ny = (x.shape[0] // la) * la, (x.shape[1] // lr) * lr
    return x[:nx, :ny].reshape(nx // la, la, ny // lr, lr).mean((1, 3))


def coherence(a, b, w1=5, w2=5):
    """|<a b*>| / sqrt(<|a|^2> <|b|^2>) over moving w1 x w2 windows in float64, the edge pixels repeated
    (fastsar/products.py:35-39, 53-67)."""
    a, b = np.asarray(a).astype(np.complex128), np.asarray(b).astype(np.complex128)

    def mov(v):
        return uniform_filter(v, (w1, w2), mode='nearest')
    x = a * np.conj(b)
    num = np.abs(mov(x.real) + 1j * mov(x.imag))
    den = np.sqrt(mov(np.abs(a) ** 2) * mov(np.abs(b) ** 2))
    return num / np.maximum(den, 1e-300)
