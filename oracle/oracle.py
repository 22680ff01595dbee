"""TEST INFRASTRUCTURE -- the oracle of the FFBP image former. Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs import this module, and only to check the CUDA path or to time the CPU baseline. The
product (fastsar_b200) never imports it.

Parity is pinned: tests/test_oracle.py checks this module's kernels and images against the reference's own outputs
(tests/golden, written by tests/golden/make_golden.py from saulpingerman/FastSAR 0.3.1).

`simulate` synthesizes point-scatterer histories on the host cores (the benchmark's reference arm, which must run no
code of the product). Two CPU implementations of the reference's factorized backprojection run through one driver
(`make_ffbp`), which restates the reference's host orchestration fastsar/ffbp_cpu.py:158-293 (level-0 children in
groups, each carried through the later levels, the float64 child phases of the deeper levels, the final-stage
geometry, the tile assembly and the crop):

  kind='port'       oracle/liboracle.so, the float64 restatement of the kernels in oracle/ffbp_oracle.c
  kind='reference'  oracle/_ref/libffbp_cpu_ref_*.so, the reference's fastsar/ffbp_cpu.cpp compiled from its own
                    sources by oracle/Makefile (AVX-512 or AVX2 build, whichever this host runs)

`backproject_fp64` is the float64 exact backprojection (fastsar/bp.py:303-348 with float64 profiles and float64
interpolation): the FP64 oracle against which the images' dB errors are stated.

The plan (tile grid, filters, float64 collection geometry) comes from fastsar_b200.plan, whose every integer and
float field tests/test_plan.py pins against the reference planner's own output.
"""
import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
C = 299792458.0
_LIBS = {}


def _host_has_avx512():
    try:
        with open('/proc/cpuinfo') as fh:
            for line in fh:
                if line.startswith('flags'):
                    return 'avx512f' in line.split()
    except OSError:
        pass
    return False


def lib_path(kind):
    if kind == 'port':
        return os.path.join(HERE, 'liboracle.so')
    if kind == 'reference':
        lvl = 'v4' if _host_has_avx512() else 'v3'
        return os.path.join(HERE, '_ref', f'libffbp_cpu_ref_{lvl}.so')
    raise ValueError(kind)


def available(kind):
    return os.path.exists(lib_path(kind))


def lib(kind='port'):
    """The kernels of `kind` as a ctypes library (built by `make -C oracle` / `make -C oracle ref`)."""
    if kind in _LIBS:
        return _LIBS[kind]
    path = lib_path(kind)
    if not os.path.exists(path):
        raise FileNotFoundError(f'{path} is missing: run make -C oracle' + (' ref' if kind == 'reference' else ''))
    L = ctypes.CDLL(path)
    f32 = np.ctypeslib.ndpointer(np.float32, flags='C_CONTIGUOUS')
    f64 = np.ctypeslib.ndpointer(np.float64, flags='C_CONTIGUOUS')
    i, dbl, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.rot_fir_k.argtypes = [f32, f32, i, i, i, f32, f32, i, f32, i, i, i, i, dbl, f32, f32]
    L.rot_fir_k_cplx.argtypes = [f32, i, i, i, f32, f32, i, f32, i, i, i, i, dbl, f32, f32]
    L.fir_p.argtypes = [f32, f32, i, i, i, f32, i, i, i, i, f32, f32]
    L.final_tiles.argtypes = [f32, f32, i, i, i, i, f64, f64, f64, f64, dbl, dbl, f64, f64, f64, dbl, f32, f32, vp, vp, vp]
    L.ffbp_cpu_threads.restype = i
    if kind == 'port':
        L.bp_points_f64.argtypes = [f64, i, i, f64, vp, f64, f64, ctypes.c_long, dbl, dbl, f64]
        L.simulate_points.argtypes = [f64, i, i, dbl, dbl, f64, f64, i, f32]
        L.simulate_points.restype = None
    _LIBS[kind] = L
    return L


# ------------------------------------------------------------------------------------------------ metrics

def rel_db(a, b):
    """10 log10 |g a - b|^2 / |b|^2 with the complex gain g fitted by least squares (the error of an image a against
    a reference b, fastsar tests/test_exact.py:20-22)."""
    a, b = np.asarray(a).ravel().astype(np.complex128), np.asarray(b).ravel().astype(np.complex128)
    g = np.vdot(a, b) / np.vdot(a, a)
    return float(10 * np.log10(np.sum(np.abs(g * a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def err_db(a, b):
    """10 log10 |a - b|^2 / |b|^2, no gain fitted (fastsar tests/test_ffbp_cpu.py:34-36)."""
    a, b = np.asarray(a).ravel().astype(np.complex128), np.asarray(b).ravel().astype(np.complex128)
    return float(10 * np.log10(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def window(P, K, sll=35.0, nbar=4):
    """The Taylor windows (-35 dB, nbar 4, unnormalised) over pulses and samples, float32 (fastsar/api.py:54-56)."""
    from scipy.signal.windows import taylor
    return (taylor(P, nbar=nbar, sll=sll, norm=False).astype(np.float32),
            taylor(K, nbar=nbar, sll=sll, norm=False).astype(np.float32))


# ------------------------------------------------------------------------------------------------ FFBP driver

def _children(L, pre, pim, c0, sl, lv):
    """One level for Np parents: pre [Np, P, K] float32 planes (or pre complex64 and pim None), c0, sl [Np, C, P]
    float32 -> [Np C, Po, Ko] float32 planes (fastsar/ffbp_cpu.py:65-103)."""
    Np, P, K = pre.shape
    Cn, Ko, Po, Dk, Dp = c0.shape[1], lv['Ko'], lv['Po'], lv['Dk'], lv['Dp']
    kc = (K - 1) / 2.0
    c0 = np.ascontiguousarray(c0, np.float32)
    sl = np.ascontiguousarray(sl, np.float32)
    if Dk > 1:
        fk = lv['fir_k']
        taps, Lk, pl = np.ascontiguousarray(fk['kern'], np.float32), fk['L'], fk['pl']
    else:
        taps, Lk, pl = np.ones(1, np.float32), 1, 0
    yre = np.empty((Np * Cn, P, Ko), np.float32)
    yim = np.empty((Np * Cn, P, Ko), np.float32)
    if Dk == 1 and L is _LIBS.get('reference'):
        # the reference rotates in NumPy float64 when nothing is decimated along frequency (fastsar/ffbp_cpu.py:87-95)
        if pim is None:
            pre, pim = np.ascontiguousarray(pre.real), np.ascontiguousarray(pre.imag)
        k = np.arange(K, dtype=np.float64) - kc
        cyc = c0[:, :, :, None].astype(np.float64) + k[None, None, None, :] * sl[:, :, :, None]
        ang = (cyc - np.rint(cyc)) * (2 * np.pi)
        cs, sn = np.cos(ang).astype(np.float32), np.sin(ang).astype(np.float32)
        yre = np.ascontiguousarray((pre[:, None] * cs - pim[:, None] * sn).reshape(Np * Cn, P, K))
        yim = np.ascontiguousarray((pre[:, None] * sn + pim[:, None] * cs).reshape(Np * Cn, P, K))
    elif pim is None:
        L.rot_fir_k_cplx(np.ascontiguousarray(pre).view(np.float32), Np, P, K, c0, sl, Cn, taps, Lk, pl, Dk, Ko, kc, yre, yim)
    else:
        L.rot_fir_k(np.ascontiguousarray(pre), np.ascontiguousarray(pim), Np, P, K, c0, sl, Cn, taps, Lk, pl, Dk, Ko, kc,
                    yre, yim)
    if Dp > 1:
        fp = lv['fir_p']
        zre = np.empty((Np * Cn, Po, Ko), np.float32)
        zim = np.empty((Np * Cn, Po, Ko), np.float32)
        L.fir_p(yre, yim, Np * Cn, P, Ko, np.ascontiguousarray(fp['kern'], np.float32), fp['L'], fp['pl'], Dp, Po, zre, zim)
        return zre, zim
    return yre, yim


def device_phases(la, refs, lv):
    """Band-centre phase and slope of every child of every parent in float64 (fastsar/ffbp_cpu.py:142-155):
    refs [Np, 3] -> c0, slope [Np, C, P] float32. The range difference is taken in the cancellation-free form
    num / (sqrt(wn^2 + num) + wn)."""
    k0c = 2.0 * (lv['f0'] + (lv['K'] - 1) / 2.0 * lv['df']) / C
    k1 = 2.0 * lv['df'] / C
    u, r0, d = la['u'], la['r0'], lv['d']
    uc = refs @ u.T
    wn = r0[None, :] * np.sqrt(1 + ((refs * refs).sum(1)[:, None] - 2 * r0[None, :] * uc) / (r0 * r0)[None, :])
    ud = d @ u.T
    wd = r0[None, None, :] * ud[None] - (d[None, :, :] * refs[:, None, :]).sum(2)[:, :, None]
    num = (d * d).sum(1)[None, :, None] - 2 * wd
    ddr = num / (np.sqrt(wn[:, None, :] ** 2 + num) + wn[:, None, :])
    c0 = ddr * k0c
    return (c0 - np.rint(c0)).astype(np.float32), (ddr * k1).astype(np.float32)


PROFILE = {}


def make_ffbp(plan, coll, kind='port', wf=None):
    """form(S [P, K] complex64, windowed) -> complex64 image [nx, ny], the reference's CPU pipeline on the kernels of
    `kind` (fastsar/ffbp_cpu.py:158-293). wf: final-subaperture weights [ntiles, Pf] or [3, ntiles, Pf]."""
    L = lib(kind)
    HOST_LEVELS = 2
    levels, T, nlev = plan['levels'], plan['T'], len(plan['levels'])
    fin = plan['final']
    Pf = fin['P']
    a0, a1, fc2 = 2.0 * fin['f0'] / C, 2.0 * fin['df'] / C, 2.0 * fin['fc'] / C
    e1, e2 = np.asarray(plan['e1'], np.float64), np.asarray(plan['e2'], np.float64)
    en = np.cross(e1, e2)
    dlx = np.ascontiguousarray((np.arange(T) - (T - 1) / 2.0) * plan['spx'], np.float64)
    dly = np.ascontiguousarray((np.arange(T) - (T - 1) / 2.0) * plan['spy'], np.float64)
    fu, fr0 = np.asarray(coll['final']['u'], np.float64), np.asarray(coll['final']['r0'], np.float64)
    fcen = np.asarray(fin['cen'], np.float64)
    sx0, sy0 = levels[0]['sx'], levels[0]['sy']
    G = sx0 * sy0
    mx, my = plan['Nx'] // sx0, plan['Ny'] // sy0
    # a level-0 child's block of final tiles, in the tile order (x1, y1, x2, y2, ..., T, T) -> [mx, my]
    shape_g = [s for lv in levels[1:] for s in (lv['sx'], lv['sy'])] + [T, T]
    perm_g = [2 * i for i in range(nlev - 1)] + [2 * (nlev - 1)] + [2 * i + 1 for i in range(nlev - 1)] + [2 * (nlev - 1) + 1]

    def final(are, aim, cen, wts=None):
        B = are.shape[0]
        w = fr0[None, :, None] * fu[None, :, :] - cen[:, None, :]
        wn = np.sqrt((w * w).sum(2))
        ux = np.ascontiguousarray((w @ e1) / wn)
        uy = np.ascontiguousarray((w @ e2) / wn)
        uz = (w @ en) / wn
        mxv, myv, mzv = ux.mean(1), uy.mean(1), uz.mean(1)
        mn = np.sqrt(mxv * mxv + myv * myv + mzv * mzv)
        ucx, ucy, rc = np.ascontiguousarray(mxv / mn), np.ascontiguousarray(myv / mn), np.ascontiguousarray(wn.mean(1))
        ore = np.empty((B, T, T), np.float32)
        oim = np.empty((B, T, T), np.float32)
        wp = [None] * 3 if wts is None else [np.ascontiguousarray(x, np.float32) for x in wts]
        L.final_tiles(np.ascontiguousarray(are), np.ascontiguousarray(aim), B, Pf, fin['K'], T, ux, uy, dlx, dly, a0, a1,
                      ucx, ucy, rc, fc2, ore, oim, *[None if x is None else x.ctypes.data for x in wp])
        return ore, oim

    def one_tile(a, b, g):
        a, b = a[None], b[None]
        for i in range(1, nlev):
            lv, la = levels[i], coll['levels'][i]
            if i < HOST_LEVELS:
                c0, sl = la['c0'][g][None], la['slope'][g][None]
            else:
                refs = np.asarray(lv['ref'], np.float64).reshape(G, a.shape[0], 3)[g]
                c0, sl = device_phases(la, refs, lv)
            a, b = _children(L, a, b, c0, sl, lv)
        cen = fcen.reshape(G, -1, 3)[g]
        if wf is not None and wf.ndim == 3:
            w = wf.reshape(3, G, -1, Pf)[:, g]
            w0 = w[0]
            gyr = np.where(np.abs(w0) > 1e-6 * max(float(np.abs(w0).max()), 1e-30), w[2] / np.where(w0 == 0, 1, w0), 0.0)
            re, im = final(a, b, cen, (w0, w[1], gyr))
        else:
            if wf is not None:
                w = wf.reshape(G, -1, Pf)[g][:, :, None]
                a, b = a * w, b * w
            re, im = final(a, b, cen)
        return (re.reshape(shape_g).transpose(perm_g).reshape(mx, my), im.reshape(shape_g).transpose(perm_g).reshape(mx, my))

    ox, oy, nx, ny = plan['ox'], plan['oy'], plan['nx'], plan['ny']

    def form(S, ng=8, children=None):
        """children: the level-0 children to form (default all); the others' pixels are left zero (a bounded
        sample of the image's work, which scales with the number of children)."""
        S = np.asarray(S)
        lv0, la0 = levels[0], coll['levels'][0]
        if S.dtype == np.complex64 and S.flags.c_contiguous and lv0['Dk'] > 1:
            pre, pim = S[None], None
        else:
            pre = np.ascontiguousarray(S.real, np.float32)[None]
            pim = np.ascontiguousarray(S.imag, np.float32)[None]
        full = np.zeros((plan['Nx'], plan['Ny']), np.complex64)
        todo = list(range(G)) if children is None else sorted(children)
        for g0 in range(0, len(todo), ng):
            gs = todo[g0:g0 + ng]
            A, Bm = _children(L, pre, pim, la0['c0'][0, gs][None], la0['slope'][0, gs][None], lv0)
            for k, g in enumerate(gs):
                re, im = one_tile(A[k], Bm[k], g)
                x, y = g // sy0, g % sy0
                full[x * mx:(x + 1) * mx, y * my:(y + 1) * my] = re + 1j * im
        return full[ox:ox + nx, oy:oy + ny].copy()

    return form


def image_former(ant, fmin, df, K, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), *, T='auto',
                 levels=None, pmax=0.4, target_db=-40.0, window_on=True, kind='port'):
    """The CPU former on the reference's defaults (fastsar/api.py:341-469, the cpu backend): T chosen by the
    predicted error, three levels unless given, the Taylor window applied in float32. -> (form(S) -> image, plan)."""
    from fastsar_b200 import plan as P_
    from fastsar_b200.sim import Collect
    ant = np.asarray(ant, np.float64)
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    if T == 'auto':
        T, _ = P_.choose_T(ant, fmin + K * df, nx, ny, spx, spy, e1, e2, target_db)
    col = Collect(fmin=float(fmin), df=float(df), K=int(K), ant=ant, res=0.5)
    nl = 3 if levels is None else levels
    while True:
        try:
            plan = P_.make_plan(col, nx, ny, spx, spy, T=T, nlev=nl, pmax=pmax, e1=e1, e2=e2)
            break
        except ValueError as e:
            if levels is not None or 'cannot split' not in str(e) or nl >= 8:
                raise
            nl += 1
    coll = P_.collection_arrays(plan, ant)
    inner = make_ffbp(plan, coll, kind)
    P = ant.shape[0]
    wp, wk = window(P, K) if window_on else (None, None)

    def form(S, ng=8, children=None):
        S = np.asarray(S)
        if window_on:
            S = (S * (wp[:, None] * wk[None, :]).astype(np.float32)).astype(np.complex64)
        else:
            S = S.astype(np.complex64)
        return inner(np.ascontiguousarray(S), ng, children)
    return form, plan


def children_mask(plan, children):
    """[nx, ny] bool: the pixels of the cropped image that the given level-0 children form."""
    sx0, sy0 = plan['levels'][0]['sx'], plan['levels'][0]['sy']
    mx, my = plan['Nx'] // sx0, plan['Ny'] // sy0
    full = np.zeros((plan['Nx'], plan['Ny']), bool)
    for g in children:
        x, y = g // sy0, g % sy0
        full[x * mx:(x + 1) * mx, y * my:(y + 1) * my] = True
    return full[plan['ox']:plan['ox'] + plan['nx'], plan['oy']:plan['oy'] + plan['ny']]


def simulate(col, pos, amp):
    """Phase history [P, K] complex64 of point scatterers on the host cores (the port's simulate_points, float64)."""
    S = np.zeros((col.Np, col.K), np.complex64)
    amp = np.ascontiguousarray(amp, np.complex128)
    lib('port').simulate_points(np.ascontiguousarray(col.ant, np.float64), col.Np, col.K, float(col.fmin),
                                float(col.df), np.ascontiguousarray(pos, np.float64), amp.view(np.float64), len(amp),
                                S.view(np.float32))
    return S


def children_pixels(plan, children):
    """Pixels of the cropped image that the given level-0 children form."""
    sx0, sy0 = plan['levels'][0]['sx'], plan['levels'][0]['sy']
    mx, my = plan['Nx'] // sx0, plan['Ny'] // sy0
    n = 0
    for g in children:
        x, y = g // sy0, g % sy0
        x0, x1 = max(x * mx, plan['ox']), min((x + 1) * mx, plan['ox'] + plan['nx'])
        y0, y1 = max(y * my, plan['oy']), min((y + 1) * my, plan['oy'] + plan['ny'])
        n += max(0, x1 - x0) * max(0, y1 - y0)
    return n


# ------------------------------------------------------------------------------------------------ FP64 exact BP

def range_compress(S, nfft):
    """S [p, K] -> [p, nfft] complex128 range profiles: zero delay at nfft // 2, the carrier of sample K // 2 removed,
    the unnormalised inverse transform (fastsar/bp.py:55-63)."""
    P, K = S.shape
    h = K // 2
    pad = np.zeros((P, nfft), np.complex128)
    pad[:, :K - h] = S[:, h:]
    pad[:, nfft - h:] = S[:, :h]
    return np.fft.fftshift(np.fft.ifft(pad, axis=1), axes=1) * nfft


def backproject_fp64(S, ant, fmin, df, points, *, rcv=None, ref=None, upsample=64, window_on=True, chunk=256):
    """Exact backprojection at points [..., 3] in float64 throughout: complex128 range profiles zero-padded
    `upsample` times (rounded up to a power of two), linear interpolation, float64 phase and accumulation
    (fastsar/bp.py:303-348). -> complex128 [...]."""
    L = lib('port')
    S = np.asarray(S)
    P, K = S.shape
    tx = np.ascontiguousarray(ant, np.float64)
    if ref is None:
        ref = np.linalg.norm(tx, axis=1) if rcv is None else 0.5 * (np.linalg.norm(tx, axis=1) + np.linalg.norm(rcv, axis=1))
    ref = np.ascontiguousarray(ref, np.float64)
    if window_on:
        wp, wk = window(P, K)
        S = S * (wp[:, None] * wk[None, :]).astype(np.float32)
    pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
    nfft = 1 << int(np.ceil(np.log2(upsample * K)))
    inv_dr = 2.0 * df * nfft / C
    kcyc = 2.0 * (fmin + (K // 2) * df) / C
    out = np.zeros(2 * len(pts))
    for p0 in range(0, P, chunk):
        sl = slice(p0, min(P, p0 + chunk))
        prof = np.ascontiguousarray(range_compress(S[sl].astype(np.complex128), nfft)).view(np.float64)
        r = None if rcv is None else np.ascontiguousarray(rcv[sl], np.float64)
        L.bp_points_f64(prof, sl.stop - sl.start, nfft, np.ascontiguousarray(tx[sl]), None if r is None else r.ctypes.data,
                        np.ascontiguousarray(ref[sl]), pts, len(pts), inv_dr, kcyc, out)
    return out.view(np.complex128).reshape(np.asarray(points).shape[:-1])


def time_cpu_former(form, S, repeats=3):
    """Best wall time of `repeats` warm calls of a CPU former on S (seconds)."""
    form(S)
    best = float('inf')
    for _ in range(repeats):
        t0 = time.perf_counter()
        form(S)
        best = min(best, time.perf_counter() - t0)
    return best
