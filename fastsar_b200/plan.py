"""FFBP plan: tile grid, decimation factors, filters and the float64 collection geometry (host side).

This is the planner of the reference's factorized backprojection, restated:

* `choose_splits`       fastsar/ffbp2.py:34-62   per-axis split factors of the levels
* `decimator_fir`       fastsar/ffbp2.py:101-137 (the kernel of fastsar/ffbp.py:57-78's Kaiser-sinc matrix)
* `decimator_shape`     fastsar/ffbp2.py:72-86   (LazyDecimator: output count and margin m)
* `make_plan`           fastsar/ffbp2.py:192-250
* `final_phase_error`   fastsar/ffbp2.py:276-297, `choose_T` fastsar/ffbp2.py:300-307
* `collection_arrays`   fastsar/ffbp2.py:313-342 (HOST_LEVELS = 2 levels of rotation phases in float64)
* `positions`           fastsar/ffbp.py:122-125
* `final_weights`       fastsar/api.py:203-244
* `plan_signature`      fastsar/ffbp2.py:259-273, `pulse_plan` fastsar/ffbp2.py:252-256
* `gate_plan`           fastsar/api.py:272-300 (the range gate), with `taper` fastsar/patches.py:156-159

Integers (splits, decimations, filter lengths and offsets, sizes) must equal the reference's exactly and floats to
1e-12: the level kernels index with them and the image's tile order depends on them. The arithmetic below follows
the reference's formulas term by term for that reason (a different but equivalent order of operations would move
the float64 results by an ulp, which is harmless, but the integer fields come from floors and ceilings of them).
"""
import functools
import math

import numpy as np

C = 299792458.0
FACTORS = (8, 7, 6, 5, 4, 3, 2)
HOST_LEVELS = 2


# ------------------------------------------------------------------------------------------------ splits

def choose_splits(n, T, nlev):
    """Smallest tile count >= ceil(n / T) that is a product of nlev non-increasing factors from FACTORS; among equal
    products the lexicographically largest factor tuple. Beyond 8**nlev, equal factors above 8 shrunk from the last
    (fastsar/ffbp2.py:34-62)."""
    need = -(-n // T)
    best = None
    stack = [((), 1)]
    while stack:
        prefix, prod = stack.pop()
        if len(prefix) == nlev:
            if prod >= need and (best is None or prod < best[0] or (prod == best[0] and prefix > best[1])):
                best = (prod, prefix)
            continue
        for f in FACTORS:
            if prefix and f > prefix[-1]:
                continue
            stack.append((prefix + (f,), prod * f))
    if best is None:
        for f in range(16, 8, -1):
            if f ** nlev >= need:
                fs = [f] * nlev
                while fs and _prod(fs[:-1]) * (fs[-1] - 1) >= need and fs[-1] > 2:
                    fs[-1] -= 1
                best = (_prod(fs), tuple(fs))
        if best is None:
            raise ValueError(f'{nlev} levels cannot split {n} pixels into tiles of {T}: use more levels or a larger T')
    return best[1]


def _prod(v):
    out = 1
    for x in v:
        out *= x
    return out


# ------------------------------------------------------------------------------------------------ filters

def _half_width(D, pass_frac, atten):
    """Kaiser design half width (input samples) of a decimation by D with passband pass_frac of the output Nyquist."""
    dw = (2.0 - 2.0 * pass_frac) * np.pi / D
    return math.ceil((atten - 8.0) / (2.285 * dw)) / 2.0 + 1.0


def decimator_shape(n_in, D, pass_frac, atten=70.0):
    """(n_out, m) of the decimation of n_in samples by D: the output grid runs m samples past each end of the input,
    output j sitting at input D (j - m) + (D - 1) / 2 (fastsar/ffbp2.py:72-86, fastsar/ffbp.py:57-78)."""
    if D == 1:
        return int(n_in), 0
    m = int(math.ceil(_half_width(D, pass_frac, atten) / D))
    return -(-int(n_in) // D) + 2 * m, m


def decimator_fir(n_in, D, pass_frac, atten=70.0):
    """The shift-invariant kernel of the Kaiser-windowed sinc decimator: dict(kern [L] float64, pl, pr, n_out, L) with
    out[j] = sum_r kern[r] x[D j + r - pl] (x zero outside [0, n_in)), and the margin m. Each column of the dense
    decimator is one windowed sinc divided by the sums of its input rows over every output (rows sum to one), so the
    kernel is the middle column's non-zero run (fastsar/ffbp2.py:101-137)."""
    d, m = _decimator_fir(int(n_in), int(D), float(pass_frac), float(atten))
    return dict(d), m


@functools.lru_cache(maxsize=512)
def _decimator_fir(n_in, D, pass_frac, atten):
    half = _half_width(D, pass_frac, atten)
    m = int(math.ceil(half / D))
    n_out = -(-n_in // D) + 2 * m
    beta = 0.1102 * (atten - 8.7)
    i0b = np.i0(beta)

    def kaiser_sinc(t):
        w = np.i0(beta * np.sqrt(np.clip(1.0 - (t / half) ** 2, 0.0, 1.0))) / i0b
        return np.where(np.abs(t) <= half, np.sinc(t / D) * w, 0.0)

    jm = n_out // 2                                       # the middle output: its column has the full support
    cm = D * (jm - m) + (D - 1) / 2.0
    idx = np.arange(max(0, int(math.floor(cm - half))), min(n_in, int(math.ceil(cm + half)) + 1))
    val = kaiser_sinc(idx - cm)
    nz = val != 0
    idx, val = idx[nz], val[nz]
    centres = D * (np.arange(n_out) - m) + (D - 1) / 2.0
    near = np.abs(centres[None, :] - idx[:, None]) <= half
    rowsum = np.where(near, kaiser_sinc(idx[:, None] - centres[None, :]), 0.0).sum(1)
    kern = val / rowsum
    L = int(idx[-1] - idx[0] + 1)
    pl = int(D * m - (int(idx[0]) - D * (jm - m)))
    assert pl >= 0 and L == len(kern)
    kern.flags.writeable = False
    pr = max(D * (n_out - 1) + L - pl - n_in, 0)
    return dict(kern=kern, pl=pl, pr=int(pr), n_out=int(n_out), L=L), m


def positions(ant, idx):
    """Antenna positions at fractional pulse indices idx, linear between pulses and extrapolated beyond the ends
    (fastsar/ffbp.py:122-125)."""
    i0 = np.clip(np.floor(idx).astype(int), 0, len(ant) - 2)
    return ant[i0] + (idx - i0)[:, None] * (ant[i0 + 1] - ant[i0])


# ------------------------------------------------------------------------------------------------ plan

def make_plan(col, nx, ny, spx, spy, T=32, nlev=3, pmax=0.4, atten=70.0, splits=None, e1=(1.0, 0.0, 0.0),
              e2=(0.0, 1.0, 0.0), pulse=None, taps=None):
    """The plan of an nx x ny image of spacings spx, spy along the orthonormal e1, e2 about the origin, for the
    collection col (fmin, df, K, ant). Returns a dict with the padded grid (Nx, Ny, ox, oy), the per-level records
    (splits sx, sy and children C; decimations Dk, Dp; sizes K, P in and Ko, Po out; filters fir_k, fir_p; the band
    f0, df of the level's input; the antenna path ant [P, 3] on the level's input pulse grid; the parents' reference
    points ref [B, 3], the child offsets d [C, 3], the child centres cen [B, C, 3], the output pulse positions pidx)
    and the final-stage record (fastsar/ffbp2.py:192-250), which adds the tiles' first pixels and the antenna path
    of the final subapertures to the reference's.
    pulse: per-level (Dp, pass_p) that replace the ones this aperture would get.
    taps: None (the reference's Kaiser-sinc decimators) or learned decimation taps (fastsar_b200.learned.LearnedTaps):
    an axis whose decimation and pass fraction the network covers takes its 8-output-sample filter (margin m = 4),
    the others keep the Kaiser-sinc one; the level records which in kind_k / kind_p."""
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    if splits is None:
        sxs, sys_ = choose_splits(nx, T, nlev), choose_splits(ny, T, nlev)
    else:
        sxs, sys_ = tuple(s[0] for s in splits), tuple(s[1] for s in splits)
    Nx, Ny = T * _prod(sxs), T * _prod(sys_)
    ox, oy = (Nx - nx) // 2, (Ny - ny) // 2
    ant = np.asarray(col.ant, np.float64)
    f0, df, K, P = float(col.fmin), float(col.df), int(col.K), int(ant.shape[0])
    ref = np.zeros((1, 3))
    first = np.zeros((1, 2))                              # first pixel index (x, y) of each parent tile
    cx, cy = Nx, Ny
    plan = dict(levels=[], T=T, nx=nx, ny=ny, Nx=Nx, Ny=Ny, ox=ox, oy=oy, spx=spx, spy=spy,
                split=list(zip(sxs, sys_)), e1=e1, e2=e2)
    for lev, (sx, sy) in enumerate(zip(sxs, sys_)):
        cx, cy = cx // sx, cy // sy
        gx, gy = np.meshgrid(np.arange(sx) * cx, np.arange(sy) * cy, indexing='ij')
        cfirst = first[:, None, :] + np.stack([gx.ravel(), gy.ravel()], axis=1)[None, :, :]       # [B, C, 2]
        cen = (((cfirst[..., 0] + (cx - 1) / 2.0 - ox - nx / 2.0) * spx)[..., None] * e1 +
               ((cfirst[..., 1] + (cy - 1) / 2.0 - oy - ny / 2.0) * spy)[..., None] * e2)
        # the child's half extent in slant range (rk) and its range change per pulse step (dop), over its corners
        u = ant / np.linalg.norm(ant, axis=1)[:, None]
        u1, u2 = u @ e1, u @ e2
        hx, hy = 0.5 * cx * spx, 0.5 * cy * spy
        rk = hx * np.abs(u1).max() + hy * np.abs(u2).max()
        dop = hx * np.abs(np.diff(u1)).max() + hy * np.abs(np.diff(u2)).max()
        kmax = 2.0 * (f0 + K * df) / C
        Dk = max(1, int(pmax * (C / (2.0 * df) / 2.0) / rk))
        Dp = max(1, int(pmax / (2.0 * kmax * dop)))
        pass_k = math.ceil(64 * rk / (C / (2.0 * df * Dk) / 2.0)) / 64
        pass_p = math.ceil(64 * 2.0 * kmax * dop * Dp) / 64
        if pulse is not None:
            Dp, pass_p = int(pulse[lev][0]), float(pulse[lev][1])
        ak, ap = min(pass_k, 0.95), min(pass_p, 0.95)
        lk = taps.decimator(K, Dk, ak, lev, 0) if taps is not None and Dk > 1 else None
        lp = taps.decimator(P, Dp, ap, lev, 1) if taps is not None and Dp > 1 else None
        Ko, mk = (lk[0]['n_out'], lk[1]) if lk else decimator_shape(K, Dk, ak, atten)
        Po, mp = (lp[0]['n_out'], lp[1]) if lp else decimator_shape(P, Dp, ap, atten)
        # an axis shorter than its decimation kernel is not decimated (late levels of small collections)
        if Dk > 1 and K < 2 * mk * Dk + Dk:
            Dk, pass_k, ak, lk = 1, rk / (C / (2.0 * df) / 2.0), 0.95, None
            Ko, mk = K, 0
        if Dp > 1 and P < 2 * mp * Dp + Dp:
            Dp, pass_p, ap, lp = 1, 2.0 * kmax * dop, 0.95, None
            Po, mp = P, 0
        pidx = Dp * (np.arange(Po) - mp) + (Dp - 1) / 2.0
        plan['levels'].append(dict(
            sx=sx, sy=sy, C=sx * sy, Dk=Dk, Dp=Dp, K=K, P=P, Ko=Ko, Po=Po, mk=mk, mp=mp,
            fir_k=(lk[0] if lk else decimator_fir(K, Dk, ak, atten)[0]) if Dk > 1 else None,
            fir_p=(lp[0] if lp else decimator_fir(P, Dp, ap, atten)[0]) if Dp > 1 else None,
            kind_k='learned' if lk else 'kaiser', kind_p='learned' if lp else 'kaiser',
            dec_k=(K, Dk, ak, taps.ident if lk else atten), dec_p=(P, Dp, ap, taps.ident if lp else atten),
            f0=f0, df=df, ant=ant, ref=ref, d=cen[0] - ref[0], cen=cen, pidx=pidx,
            pass_k=float(pass_k), pass_p=float(pass_p)))
        ant = positions(ant, pidx)
        f0, df, K, P = f0 + ((Dk - 1) / 2.0 - mk * Dk) * df, df * Dk, Ko, Po
        ref, first = cen.reshape(-1, 3), cfirst.reshape(-1, 2)
    assert (cx, cy) == (T, T)
    # first: the first pixel (x, y) of each final tile on the padded grid, in the tile order of cen
    plan['final'] = dict(cen=ref, first=first.astype(np.int64), f0=f0, df=df, K=K, P=P, fc=f0 + (K - 1) / 2.0 * df,
                         ant=ant)
    return plan


def pulse_plan(plan):
    """Per-level (Dp, pass_p) of a plan and the product of its pulse decimations (fastsar/ffbp2.py:252-256)."""
    return [(lv['Dp'], lv['pass_p']) for lv in plan['levels']], _prod(lv['Dp'] for lv in plan['levels'])


def plan_signature(plan):
    """The shape-defining constants of a plan as a hashable tuple: equal signatures mean equal launch shapes and
    filters (fastsar/ffbp2.py:259-273)."""
    lv = []
    for l in plan['levels']:
        fk = l['fir_k'] and (l['fir_k']['L'], l['fir_k']['pl'], l['fir_k']['pr'], l['fir_k']['n_out'])
        fp = l['fir_p'] and (l['fir_p']['L'], l['fir_p']['pl'], l['fir_p']['pr'], l['fir_p']['n_out'])
        lv.append((l['sx'], l['sy'], l['C'], l['Dk'], l['Dp'], l['K'], l['P'], l['Ko'], l['Po'], float(l['f0']),
                   float(l['df']), fk, fp, l['dec_k'], l['dec_p'], l['pass_k'], l['pass_p']))
    f = plan['final']
    return (tuple(lv), (f['P'], f['K'], float(f['f0']), float(f['df']), float(f['fc'])), plan['T'], plan['nx'],
            plan['ny'], plan['Nx'], plan['Ny'], plan['ox'], plan['oy'], float(plan['spx']), float(plan['spy']),
            tuple(map(float, plan['e1'])), tuple(map(float, plan['e2'])))


# ------------------------------------------------------------------------------------------------ final tile size

def final_phase_error(ant, fmax, nx, ny, spx, spy, e1, e2, T):
    """Predicted image error (dB) of the final stage's plane-wave-plus-mean-curvature model on T x T tiles: the peak
    residual range over pulses, tile corners and a 3 x 3 sample of tile positions, as a phase at fmax, mapped by
    20 log10(phase) - 14 dB (fastsar/ffbp2.py:276-297)."""
    ant, e1, e2 = np.asarray(ant, np.float64), np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    a = ant[::max(1, len(ant) // 2048)]
    hx, hy = 0.5 * T * spx, 0.5 * T * spy
    worst = 1e-30
    for fx in (-0.5, 0.0, 0.5):
        for fy in (-0.5, 0.0, 0.5):
            c = fx * max(0.0, nx * spx - 2 * hx) * e1 + fy * max(0.0, ny * spy - 2 * hy) * e2
            w = a - c
            r = np.linalg.norm(w, axis=1)
            u = w / r[:, None]
            for sx in np.linspace(-1, 1, 5):
                for sy in np.linspace(-1, 1, 5):
                    d = sx * hx * e1 + sy * hy * e2
                    ud = u @ d
                    res = np.linalg.norm(w - d, axis=1) - r + ud - (d @ d - ud * ud).mean() / (2 * r.mean())
                    worst = max(worst, float(np.abs(res - res.mean()).max()))
    return 20.0 * np.log10(4 * np.pi * fmax / C * worst) - 14.0


def choose_T(ant, fmax, nx, ny, spx, spy, e1, e2, target_db=-40.0, choices=(32, 16)):
    """The largest final tile size whose predicted error meets target_db (else the smallest), with its prediction
    (fastsar/ffbp2.py:300-307)."""
    err = None
    for T in choices:
        err = final_phase_error(ant, fmax, nx, ny, spx, spy, e1, e2, T)
        if err <= target_db:
            return T, err
    return choices[-1], err


# ------------------------------------------------------------------------------------------------ range gate

def taper(f, band, guard):
    """1 over the band, a raised cosine to 0 across the guard on either side (fastsar/patches.py:156-159)."""
    t = np.clip(np.maximum(band[0] - f, f - band[1]) / guard, 0, 1)
    return 0.5 * (1 + np.cos(np.pi * t))


def gate_plan(ant, ref, fmin, df, K, nx, ny, spx, spy, e1, e2):
    """The range gate of an nx x ny image centred on the origin (fastsar/api.py:272-300): the spectrum padded by a
    guard of an eighth of the band on either side (npl samples below, Kp in all, a fast FFT length), each pulse's
    inverse transform cut to the N range bins about its reference range that the image's points span over the
    aperture (sampled at up to 257 pulses) with a margin of 6 range resolutions of the guard, and the transform back
    kept over the band and its guards (samples k0 .. k1 - 1 of N), tapered to 0 across the guards. -> dict(npl, Kp,
    N, k0, k1, taper [k1 - k0] float32 (with the scale Kp / N), fmin, df: of the gated history)."""
    from scipy.fft import next_fast_len
    ant = np.asarray(ant, np.float64)
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    band = (fmin, fmin + (K - 1) * df)
    guard = 0.125 * (band[1] - band[0])
    npl = int(np.ceil(guard / df))
    Kp = next_fast_len(K + 2 * npl)
    idx = np.unique(np.linspace(0, len(ant) - 1, min(len(ant), 257)).astype(np.int64))
    a = ant[idx]
    r0 = np.linalg.norm(a, axis=1) if ref is None else np.asarray(ref, np.float64)[idx]
    t = np.linspace(-0.5, 0.5, 5)
    pts = ((t * nx * spx)[:, None, None] * e1 + (t * ny * spy)[None, :, None] * e2).reshape(-1, 3)
    half = np.abs(np.linalg.norm(pts[None] - a[:, None], axis=2) - r0[:, None]).max() + 6 * C / (2 * guard)
    N = next_fast_len(2 * int(np.ceil(half * 2 * Kp * df / C)))
    N += N % 2
    df2, f0 = Kp * df / N, fmin - npl * df
    T = taper(f0 + df2 * np.arange(N), band, guard)
    keep = np.nonzero(T > 0)[0]
    k0, k1 = int(keep[0]), int(keep[-1]) + 1
    return dict(npl=npl, Kp=int(Kp), N=int(N), k0=k0, k1=k1, taper=(T[k0:k1] * (Kp / N)).astype(np.float32),
                fmin=float(f0 + k0 * df2), df=float(df2))


# ------------------------------------------------------------------------------------------------ geometry

def collection_arrays(plan, ant, ref=None):
    """Per-collection float64 geometry: per level the antenna path on the level's input pulse grid as unit vectors u
    [P, 3] and ranges r0 [P]; for the first HOST_LEVELS levels also the rotation phase of every child at band centre,
    wrapped to [-0.5, 0.5] cycles (c0) and its slope in cycles per frequency sample (slope), [B, C, P] float32.
    ref [P]: the one-way range each pulse is referenced to when it is not |ant| (fastsar/ffbp2.py:313-342)."""
    ant = np.asarray(ant, np.float64)
    out = dict(levels=[])
    for i, lv in enumerate(plan['levels']):
        r0 = np.linalg.norm(ant, axis=1)
        e = dict(u=ant / r0[:, None], r0=r0)
        if i < HOST_LEVELS:
            kc = (lv['K'] - 1) / 2.0
            B, Cn = lv['ref'].shape[0], lv['C']
            c0 = np.empty((B, Cn, lv['P']), np.float32)
            sl = np.empty((B, Cn, lv['P']), np.float32)
            kcen = 2.0 * (lv['f0'] + kc * lv['df']) / C
            kstep = 2.0 * lv['df'] / C
            for b in range(B):
                base = np.linalg.norm(lv['ref'][b][None, :] - ant, axis=1)
                if i == 0 and ref is not None:
                    base = np.asarray(ref, np.float64)
                ddr = np.linalg.norm(lv['cen'][b][:, None, :] - ant[None, :, :], axis=2) - base[None, :]
                cyc = kcen * ddr
                c0[b] = cyc - np.round(cyc)
                sl[b] = kstep * ddr
            e['c0'], e['slope'] = c0, sl
        out['levels'].append(e)
        ant = positions(ant, lv['pidx'])
    r0 = np.linalg.norm(ant, axis=1)
    out['final'] = dict(u=ant / r0[:, None], r0=r0)
    return out


def final_weights(plan, weight, P, grad=False, points=None, nodes=3, first=0):
    """Mean aperture weight of each final subaperture at each final tile [ntiles, Pf] float32 (with grad=True the
    weight and its gradients along e1 and e2 per metre, [3, ntiles, Pf]): weight(points [m, 3], pulses [n]) -> [n, m]
    averaged over the input pulses a final subaperture spans by 3-point Gauss-Legendre quadrature (nodes=1: its
    centre pulse). `first`: the collection is the P pulses from pulse `first` of the plan's (fastsar/api.py:203-244)."""
    if nodes not in (1, 3):
        raise ValueError(f'final_weights: nodes must be 1 or 3, got {nodes!r}')
    cen = np.asarray(plan['final']['cen'], np.float64)
    if grad:
        h1, h2 = 0.5 * plan['T'] * plan['spx'], 0.5 * plan['T'] * plan['spy']
        e1, e2 = np.asarray(plan['e1'], np.float64), np.asarray(plan['e2'], np.float64)
        w0 = final_weights(plan, weight, P, points=cen, first=first)
        m = len(cen)
        pts = np.concatenate([cen + h1 * e1, cen - h1 * e1, cen + h2 * e2, cen - h2 * e2])
        wq = final_weights(plan, weight, P, points=pts, nodes=1, first=first)
        return np.stack([w0, (wq[:m] - wq[m:2 * m]) / (2 * h1), (wq[2 * m:3 * m] - wq[3 * m:]) / (2 * h2)]).astype(np.float32)
    q = cen if points is None else points
    idx, D = np.arange(plan['final']['P'], dtype=np.float64), 1.0
    for lv in reversed(plan['levels']):
        idx = lv['Dp'] * idx + float(lv['pidx'][0])
        D *= lv['Dp']
    a = np.clip(idx - D / 2, first - 0.5, first + P - 0.5)
    b = np.clip(idx + D / 2, first - 0.5, first + P - 0.5)
    if nodes == 1:
        t, gw = np.array([0.0]), np.array([1.0])
    else:
        t, gw = np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)]), np.array([5.0, 8.0, 5.0]) / 18.0
    nd = np.clip(np.rint(0.5 * (a + b)[:, None] + 0.5 * (b - a)[:, None] * t[None, :]), first, first + P - 1).astype(np.int64)
    U, inv = np.unique(nd.ravel(), return_inverse=True)
    W = np.asarray(weight(q, U), np.float64)[inv].reshape(len(idx), len(t), -1)
    acc = gw[0] * W[:, 0]
    for k in range(1, len(t)):
        acc = acc + gw[k] * W[:, k]
    return np.ascontiguousarray(acc.T, np.float32)
