"""Generate the golden fixtures under tests/golden from the reference implementation (saulpingerman/FastSAR 0.3.1).

Run where the reference's sources are present, naming their directory by --ref or the FASTSAR_REFERENCE environment
variable:

    FASTSAR_REFERENCE=<reference checkout> python tests/golden/make_golden.py [--only exact|gate|weights]

The reference's modules fastsar/ffbp.py and fastsar/ffbp2.py import JAX at module level but its planner and CPU paths
use only NumPy, so a stub `jax` package is inserted before the import; its C++ kernels are compiled by its own
fastsar/_build.py with the system g++ (CXX=/usr/bin/g++, which has libgomp). Nothing here is needed at test time:
the tests read only the .npz files this writes.

Fixtures:
  plan_<case>.npz     make_plan / choose_T / collection_arrays of a geometry (integers exact, floats to 1e-12)
  fir.npz             decimator_fir kernels for a spread of (n_in, D, pass) values
  kernels.npz         the reference C++ kernels rot_fir_k_cplx, rot_fir_k, fir_p, final_tiles on seeded small inputs
  image_<case>.npz    ImageFormer(backend='cpu') images (history, image), ExactFormer(cpu) and backproject(cpu, 64x)
  exact_setup.npz     ExactFormer's set-up (tile, centres, reachable bins) on geometries that pick 32 x 32 and 16 x 16
                      tiles (python tests/golden/make_golden.py --only exact writes this file alone)
  gate.npz            the range gate: _gate_plan on wide-band and spotlight geometries, the gated history of a seeded
                      random history (first pulses), and ImageFormer(backend='cpu', range_gate=True)'s image of a
                      simulated wide-band scene (python tests/golden/make_golden.py --only gate writes this file alone)
  stack.npz           the stack products: registration (_detected, _peak, _estimate), translation (_translate),
                      incoherent average (_Mean, _level) and products.multilook / interferogram / coherence of three
                      seeded images (stack_scene below; --only stack writes this file alone)
  mosaic.npz          the patch mosaic: form_mosaic (backend='cpu') on mosaic_scene's history in four cases (all
                      pulses; a beam and a Hann azimuth window; one patch; uneven patches at T = 16 and 2 levels), the
                      patch history of one patch with and without shared range profiles, and the helpers tile_plan,
                      _levels, beam_span, fill_gaps, choose_buckets (--only mosaic writes this file alone)
  weights.npz         aperture weights: api.final_weights (plain and with gradients) of the test scene's 2-level plan
                      for a pixel- and pulse-dependent weight (WEIGHT below), and ImageFormer(backend='cpu',
                      aperture_weight=WEIGHT)'s image (--only weights writes this file alone)
"""
import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def import_reference(path):
    os.environ['CXX'] = '/usr/bin/g++'
    os.environ.setdefault('FASTSAR_CACHE_DIR', '/tmp/fastsar_golden_cache')
    jax = types.ModuleType('jax')
    jnp = types.ModuleType('jax.numpy')
    lax = types.ModuleType('jax.lax')

    class Precision:
        HIGHEST, HIGH, DEFAULT = 'highest', 'high', None
    lax.Precision = Precision
    jax.numpy, jax.lax = jnp, lax
    jax.jit = lambda f=None, **k: (f if f is not None else (lambda g: g))
    jax.devices = lambda *a, **k: []
    sys.modules.update({'jax': jax, 'jax.numpy': jnp, 'jax.lax': lax})
    sys.path.insert(0, path)
    import fastsar  # noqa: F401
    return fastsar


def stats(a):
    """Summary of a large float array: count, sum, sum of squares, a strided sample (fixture size stays small)."""
    a = np.asarray(a, np.float64).ravel()
    step = max(1, len(a) // 4096)
    return np.concatenate([[len(a), a.sum(), (a * a).sum()], a[::step]])


def plan_record(ffbp2, col, nx, ny, spx, spy, e1, e2, T, nlev, pmax=0.4, full_limit=30000):
    plan = ffbp2.make_plan(col, nx, ny, spx, spy, T=T, nlev=nlev, pmax=pmax, e1=e1, e2=e2)
    rec = dict(ant=col.ant, scal=np.array([col.fmin, col.df, col.K, nx, ny, spx, spy, T, nlev, pmax], np.float64),
               e1=np.asarray(e1, np.float64), e2=np.asarray(e2, np.float64),
               top=np.array([plan['T'], plan['Nx'], plan['Ny'], plan['ox'], plan['oy']], np.int64),
               nlevels=np.array(len(plan['levels'])))
    for i, l in enumerate(plan['levels']):
        fk, fp = l['fir_k'], l['fir_p']
        rec[f'lv{i}_ints'] = np.array([l['sx'], l['sy'], l['C'], l['Dk'], l['Dp'], l['K'], l['P'], l['Ko'], l['Po'],
                                       fk['L'] if fk else -1, fk['pl'] if fk else -1, fk['pr'] if fk else -1,
                                       fk['n_out'] if fk else -1, fp['L'] if fp else -1, fp['pl'] if fp else -1,
                                       fp['pr'] if fp else -1, fp['n_out'] if fp else -1], np.int64)
        rec[f'lv{i}_f'] = np.array([l['f0'], l['df'], l['pass_k'], l['pass_p'], l['Fk'].args[2], l['Fp'].args[2]])
        if fk:
            rec[f'lv{i}_kk'] = np.asarray(fk['kern'])
        if fp:
            rec[f'lv{i}_kp'] = np.asarray(fp['kern'])
        for key in ('cen', 'd', 'ref', 'pidx'):
            a = np.asarray(l[key], np.float64)
            rec[f'lv{i}_{key}'] = a if a.size <= full_limit else stats(a)
    f = plan['final']
    rec['final_f'] = np.array([f['P'], f['K'], f['f0'], f['df'], f['fc']], np.float64)
    rec['final_cen'] = f['cen'] if f['cen'].size <= full_limit else stats(f['cen'])
    fmax = col.fmin + col.K * col.df
    Tc, err = ffbp2.choose_T(col.ant, fmax, nx, ny, spx, spy, np.asarray(e1, float), np.asarray(e2, float))
    rec['choose_T'] = np.array([Tc, err])
    rec['phase_err'] = np.array([ffbp2.final_phase_error(col.ant, fmax, nx, ny, spx, spy, np.asarray(e1, float),
                                                         np.asarray(e2, float), t) for t in (16, 32)])
    coll = ffbp2.collection_arrays(plan, col.ant)
    for i, c in enumerate(coll['levels']):
        for key in ('u', 'r0', 'c0', 'slope'):
            if key in c:
                a = np.asarray(c[key])
                rec[f'ca{i}_{key}'] = a if a.size <= full_limit else stats(a)
    rec['caf_u'] = coll['final']['u'] if coll['final']['u'].size <= full_limit else stats(coll['final']['u'])
    rec['caf_r0'] = coll['final']['r0'] if coll['final']['r0'].size <= full_limit else stats(coll['final']['r0'])
    return plan, coll, rec


def exact_setup(sim, ExactFormer):
    """ExactFormer(backend='cpu')'s geometry-only set-up: the tile, the tile centres, the window of bins per pulse."""
    rec = {}
    cases = {'r5k': (sim.make_collect(res=0.5, scene=60.0, r0=5e3), 128, 128, 0.5, 0.5),
             'r1k': (sim.make_collect(res=0.5, scene=60.0, r0=1e3), 96, 80, 0.5, 0.5),
             'wide': (sim.make_collect(res=0.3, scene=100.0, r0=2e4), 300, 200, 0.3, 0.25)}
    for name, (col, nx, ny, spx, spy) in cases.items():
        f = ExactFormer(col.ant, col.fmin, col.df, col.K, nx, ny, spx, spy, backend='cpu')
        rec[f'{name}_ant'] = col.ant
        rec[f'{name}_scal'] = np.array([col.fmin, col.df, col.K, nx, ny, spx, spy], np.float64)
        rec[f'{name}_tile'] = np.array(f.tile, np.int64)
        rec[f'{name}_err'] = np.array(f.predicted_error_db)
        rec[f'{name}_cen'] = f.cen
        rec[f'{name}_blo'] = np.asarray(f.blo, np.int64)
        rec[f'{name}_W'] = np.array(f.W, np.int64)
        rec[f'{name}_nfft'] = np.array(f.nfft, np.int64)
        rec[f'{name}_inv_dr'] = np.array(f.inv_dr)
        rec[f'{name}_kcyc'] = np.array(f.kcyc)
        print('exact setup', name, f.tile, f.W, f.nfft)
    np.savez_compressed(os.path.join(HERE, 'exact_setup.npz'), **rec)


def wide_band_collection(sim_mod, K=24000, P=384):
    """An image narrow in range from a wide-band collection (the reference's wide_band case of tests/test_api.py:
    0.5 m resolution, 30 km, 40 deg grazing)."""
    res, r0 = 0.5, 30e3
    df = 299792458.0 / (2 * res) / K
    y = (np.arange(P) - (P - 1) / 2) * (r0 * 299792458.0 / 9.6e9 / (2 * res) / P)
    psi = np.radians(40.0)
    ant = np.stack([np.full(P, -r0 * np.cos(psi)), y, np.full(P, r0 * np.sin(psi))], 1)
    return sim_mod.Collect(fmin=9.6e9 - (K // 2) * df, df=df, K=K, ant=ant, res=res)


def wide_band_scene(seed=3):
    """5 bright points in the 96 x 96 image at 0.4 m and 200 clutter scatterers over 3 km of range around it."""
    rng = np.random.default_rng(seed)
    pts = np.array([[0.0, 0.0, 0], [11.3, -7.1, 0], [-14.2, 12.4, 0], [15.1, 16.2, 0], [-9.3, -15.7, 0]])
    cl = np.stack([(rng.random(200) - 0.5) * 3000, (rng.random(200) - 0.5) * 60, np.zeros(200)], 1)
    amp = np.concatenate([np.full(5, 30.0), (rng.standard_normal(200) + 1j * rng.standard_normal(200)) / np.sqrt(2)])
    return np.concatenate([pts, cl]), amp


def gate(fastsar):
    """The range gate's plan, gated history and a gated image from the reference (fastsar/api.py:272-300, 525-564)."""
    from fastsar import sim, api
    from fastsar_b200 import sim as mysim
    rec = {}
    col = wide_band_collection(sim)
    grid = dict(nx=96, ny=96, spx=0.4, spy=0.4, e1=(0.0, 1.0, 0.0), e2=(1.0, 0.0, 0.0))
    w4 = mysim.workload('spotlight_4k')
    cases = {'wide': (col, None, grid),
             'wide_ref': (col, np.linalg.norm(col.ant, axis=1) + 3.0, grid),
             'wide_rect': (col, None, dict(nx=160, ny=48, spx=0.3, spy=0.5, e1=(0.0, 1.0, 0.0), e2=(1.0, 0.0, 0.0))),
             'spot4k': (w4['col'], None, dict(nx=256, ny=256, spx=0.25, spy=0.25, e1=w4['e1'], e2=w4['e2']))}
    for name, (c, ref, g) in cases.items():
        gp = api._gate_plan(c.ant, ref, float(c.fmin), float(c.df), c.K, g['nx'], g['ny'], g['spx'], g['spy'],
                            np.asarray(g['e1'], float), np.asarray(g['e2'], float))
        rec[f'{name}_ant'] = c.ant
        rec[f'{name}_ref'] = np.zeros(0) if ref is None else ref
        rec[f'{name}_scal'] = np.array([c.fmin, c.df, c.K, g['nx'], g['ny'], g['spx'], g['spy']], np.float64)
        rec[f'{name}_e'] = np.array([g['e1'], g['e2']], np.float64)
        rec[f'{name}_ints'] = np.array([gp['npl'], gp['Kp'], gp['N'], gp['k0'], gp['k1']], np.int64)
        rec[f'{name}_fl'] = np.array([gp['fmin'], gp['df']])
        rec[f'{name}_taper'] = gp['taper']
        print('gate plan', name, rec[f'{name}_ints'])
    # the gated history of a seeded random history (windowed), its first 8 pulses
    args = (col.ant, col.fmin, col.df, col.K)
    f = api.ImageFormer(*args, **grid, backend='cpu', range_gate=True)
    rng = np.random.default_rng(21)
    S = (rng.standard_normal((col.ant.shape[0], col.K)) + 1j * rng.standard_normal((col.ant.shape[0], col.K))).astype(np.complex64)
    rec['hist_gated'] = np.asarray(f._gate(S))[:8]
    rec['hist_kept'] = np.array(f.range_gate['kept'])
    # a gated image of a simulated scene (float64 direct sum on the host)
    pos, amp = wide_band_scene()
    S = mysim.simulate_brute(wide_band_collection(mysim), pos, amp).astype(np.complex64)
    rec['img_pos'], rec['img_amp'] = pos, amp
    rec['img'] = f(S)
    rec['img_levels'] = np.array(f.levels)
    rec['img_Dk0'] = np.array(f._plan['levels'][0]['Dk'])
    print('gated image', rec['img'].shape, 'kept', f.range_gate['kept'], 'levels', f.levels)
    np.savez_compressed(os.path.join(HERE, 'gate.npz'), **rec)


def weight_fn(P):
    """The aperture weight of the weights fixture: weight(points [m, 3], pulses [n]) -> [n, m], a raised cosine over
    the pulses times a gentle linear ramp over the scene (pixel-dependent, so the gradient terms matter).
    tests/test_plan.py and tests/test_gpu_weights.py build the same function."""
    def w(q, p):
        q, p = np.asarray(q, np.float64), np.asarray(p, np.float64)
        over_p = 0.55 + 0.45 * np.cos(np.pi * (p - 0.5 * (P - 1)) / P)
        over_q = 1.0 + 0.006 * q[:, 0] - 0.004 * q[:, 1]
        return over_p[:, None] * over_q[None, :]
    return w


def weights(fastsar):
    """weights.npz: the reference's final_weights and its CPU former's image with an aperture weight."""
    from fastsar import sim, ffbp2, api
    c_small = sim.make_collect(res=0.5, scene=60.0, r0=5e3)
    rng = np.random.default_rng(1)                                 # the scene of fastsar tests/test_ffbp_cpu.py
    pos = np.stack([rng.uniform(-25, 25, 40), rng.uniform(-25, 25, 40), np.zeros(40)], 1)
    amp = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    S = sim.simulate_brute(c_small, pos, amp).astype(np.complex64)
    P = S.shape[0]
    wfun = weight_fn(P)
    plan = ffbp2.make_plan(c_small, 128, 128, 0.5, 0.5, T=16, nlev=2, pmax=0.4, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0))
    # the history is image_small.npz's (the same seeded scene), so it is not stored again
    rec = dict(w_plain=api.final_weights(plan, wfun, P), w_grad=api.final_weights(plan, wfun, P, grad=True),
               w_centre=api.final_weights(plan, wfun, P, nodes=1))
    for nlev in (2, 3):
        f = api.ImageFormer(c_small.ant, c_small.fmin, c_small.df, c_small.K, 128, 128, 0.5, 0.5, backend='cpu', T=16,
                            levels=nlev, window=False, aperture_weight=wfun)
        rec[f'img_l{nlev}'] = f(S)
    np.savez_compressed(os.path.join(HERE, 'weights.npz'), **rec)
    print('weights done', rec['w_grad'].shape)


def stack_scene(n1=128, n2=160, seed=20261204):
    """Three seeded complex images of one speckle scene on a common grid (band-limited to 0.35 of the sampling rate
    along both axes, 12 bright points): a; b, the scene displaced by (3.3, -2.6) pixels (b(x) = a(x + d)) at 0.95
    of a's amplitude plus an independent speckle at 0.3; c, an independent scene 1.7 times as bright with an
    unprocessed (zero) corner of 8 x 10 pixels."""
    rng = np.random.default_rng(seed)
    k1, k2 = np.fft.fftfreq(n1)[:, None], np.fft.fftfreq(n2)[None, :]
    band = (np.abs(k1) < 0.35) & (np.abs(k2) < 0.35)

    def white():
        w = (rng.standard_normal((n1, n2)) + 1j * rng.standard_normal((n1, n2))) / np.sqrt(2.0)
        i, j = rng.integers(8, n1 - 8, 12), rng.integers(8, n2 - 8, 12)
        w[i, j] += 8.0 * np.exp(2j * np.pi * rng.random(12))
        return np.fft.fft2(w)

    def image(F, d=(0.0, 0.0)):
        return np.fft.ifft2(F * band * np.exp(2j * np.pi * (k1 * d[0] + k2 * d[1])))
    F0, F1, F2 = white(), white(), white()
    a = image(F0).astype(np.complex64)
    b = (0.95 * image(F0, (3.3, -2.6)) + 0.3 * image(F1)).astype(np.complex64)
    c = (1.7 * image(F2)).astype(np.complex64)
    c[:8, :10] = 0
    return a, b, c


def stack(fastsar):
    """stack.npz: the reference's registration, translation and incoherent average (fastsar/stack.py) and its
    multilook, interferogram and coherence (fastsar/products.py) on stack_scene's images."""
    from fastsar import stack as st, products as pr
    a, b, c = stack_scene()
    rec = dict(a=a, b=b, c=c)
    rec['box5_a'] = st._box(st._power(a), 5)
    rec['box4_c'] = st._box(st._power(c), 4)
    da, db = st._detected(a, 5), st._detected(b, 5)
    rec['det_a'], rec['det_b'] = da, db
    rec['det3_c'] = st._detected(c, 3)
    for tag, hp in (('hp', 32.0), ('nohp', None)):
        e = st._estimate(da, db, 0.25, 0.3, 16, 2, hp)
        for k in ('shift_px', 'shift', 'significance', 'correlation', 'found', 'tiles', 'tiles_used', 'tile_residuals',
                  'tile_used', 'tile_significance', 'residual_rms', 'residual_median', 'residual_worst'):
            rec[f'est_{tag}_{k}'] = np.asarray(e[k])
        d, z, rho, clear = st._peak(da, db, 16, highpass=hp)
        rec[f'peak_{tag}'] = np.array([d[0], d[1], z, rho, float(clear)])
    # a peak searched about a given translation with a narrow window, as the tiles are
    d, z, rho, clear = st._peak(da[:64, :80], db[:64, :80], 16, around=(-3, 3), narrow=8)
    rec['peak_tile'] = np.array([d[0], d[1], z, rho, float(clear)])
    pb = st._power(b)
    rec['tr_real'] = st._translate(pb, (1.3, -0.4))
    rec['tr_cplx'] = st._translate(c, (2.25, -1.5))
    rec['tr_whole'] = st._translate(c, (-3.0, 2.0))
    # the average: of the three small complex images (too small for the looks), and of a 256 x 256 scene given as
    # one complex image and two amplitude (real) images
    a2, b2, c2 = stack_scene(256, 256, seed=20261205)
    b2, c2 = np.abs(b2).astype(np.float32), np.abs(c2).astype(np.float32)
    rec.update(m_a=a2, m_b=b2, m_c=c2)
    for tag, eq, w, imgs in (('small', None, (1.0, 2.0, 0.5), (a, b, c)), ('plain', None, (1.0, 2.0, 0.5), (a2, b2, c2)),
                             ('mean', 'mean', (1.0, 1.0, 1.0), (a2, b2, c2)),
                             ('median', 'median', (1.0, 0.5, 2.0), (a2, b2, c2))):
        acc = st._Mean(eq, 32)
        for img, wk in zip(imgs, w):
            acc.add(dict(image=img), wk)
        M = acc.image()
        L = acc.looks(M)
        rec[f'mean_{tag}_M'] = M
        rec[f'mean_{tag}_gains'] = np.array(acc.gains)
        rec[f'mean_{tag}_weights'] = np.array(w)
        for k in ('looks', 'looks_single', 'looks_by_n', 'looks_ideal', 'looks_independent', 'brightness_spread_db',
                  'tiles_selected', 'homogeneous'):
            v = L.get(k)
            rec[f'mean_{tag}_{k}'] = np.asarray(np.nan if v is None else v)
    rec['level_mean'] = np.array(st._level(st._power(c), 'mean'))
    rec['level_median'] = np.array(st._level(st._power(c), 'median'))
    rec['ml_a_2_3'] = pr.multilook(a, 2, 3)
    rec['ifg_ab_2_2'] = pr.interferogram(a, b, 2, 2)
    rec['coh_ab_5_5'] = pr.coherence(a, b, 5, 5)
    rec['coh_ac_7_3'] = pr.coherence(a, c, 7, 3)
    rec['coh_ab_4_6'] = pr.coherence(a, b, 4, 6)
    np.savez_compressed(os.path.join(HERE, 'stack.npz'), **rec)
    print('stack done', rec['est_hp_shift_px'], rec['peak_hp'], rec['mean_plain_looks'], rec['mean_median_gains'])


def mosaic_scene(seed=20261206):
    """A small collection for the mosaic fixtures: the reference's make_collect (0.5 m, 80 m scene, 5 km, 30 deg
    grazing), 24 unit points of seeded phases in a 60 m square, simulated by direct sum; the FX history with its
    reference ranges |a_p| and band. -> (collect, fx, beam): beam(idx, points) the normalized along-track offset of
    the points seen from pulses idx, 1 at 20 m (a stripmap-like footprint of 40 m)."""
    from fastsar import sim
    rng = np.random.default_rng(seed)
    col = sim.make_collect(res=0.5, scene=80.0, r0=5e3, graze_deg=30.0)
    pos = np.c_[rng.uniform(-30.0, 30.0, (24, 2)), np.zeros(24)]
    amp = np.exp(2j * np.pi * rng.random(24))
    S = sim.simulate_brute(col, pos, amp).astype(np.complex64)
    fx = dict(S=S, fmin=float(col.fmin), df=float(col.df), ref=np.linalg.norm(col.ant, axis=1),
              band=(float(col.fmin), float(col.fmin + (col.K - 1) * col.df)))
    ant = np.asarray(col.ant, np.float64)

    def beam(idx, pts):
        d = np.asarray(pts, np.float64)[None, :, :] - ant[np.asarray(idx)][:, None, :]
        return d[..., 1] / 20.0
    return col, fx, beam


def mosaic_pulses(center):
    """The mosaic fixtures' pulse span as a function of a patch centre: 150 pulses about the track point abeam of it
    (the collection's 284 pulses are 0.55 m apart along y)."""
    mid = int(round(142 + float(center[1]) / 0.55))
    return max(0, mid - 75), min(284, mid + 75)


def mosaic(fastsar):
    """mosaic.npz: the reference's patch mosaic (fastsar/patches.py form_mosaic with backend='cpu') on mosaic_scene,
    its patch histories (patch_history with and without shared range profiles) and its host helpers."""
    from fastsar import patches
    col, fx, beam = mosaic_scene()
    ant = np.asarray(col.ant, np.float64)
    e1, e2 = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)
    origin = np.array([-32.0, -32.0, 0.0])
    rec = dict(S=fx['S'], fmin=fx['fmin'], df=fx['df'], ref=fx['ref'], band=np.array(fx['band']), ant=ant,
               origin=origin)
    cases = dict(
        a=dict(nx=128, ny=128, patch=(64, 64), crop=8),
        b=dict(nx=128, ny=128, patch=(64, 64), crop=8, beam=beam, umax=1.0, awin='hann'),
        c=dict(nx=64, ny=64, patch=(64, 64), crop=0),
        d=dict(nx=96, ny=128, patch=(48, 64), crop=4, beam=beam, umax=1.0, T=16, levels=2),
    )
    # dropped pulses (filled by zero pulses at their positions), and pulses chosen by a function of the patch centre
    keep = np.setdiff1d(np.arange(len(ant)), [100, 101, 102, 170])
    fx_gap = dict(fx, S=fx['S'][keep], ref=fx['ref'][keep])
    rec['gap_keep'] = keep
    cases['e'] = dict(nx=128, ny=128, patch=(64, 64), crop=8, fx=fx_gap, ant=ant[keep])
    cases['f'] = dict(nx=128, ny=128, patch=(64, 64), crop=8, pulses=mosaic_pulses)
    for tag, kw in cases.items():
        info = []
        kw = dict(kw)
        nx, ny = kw.pop('nx'), kw.pop('ny')
        fxc, antc = kw.pop('fx', fx), kw.pop('ant', ant)
        img = patches.form_mosaic(fxc, antc, origin, nx, ny, 0.5, 0.5, e1, e2, backend='cpu', info=info, **kw)
        rec[f'img_{tag}'] = img
        rec[f'info_{tag}'] = np.array([[i['pulses'][0], i['pulses'][1], i['K'], i['T'], i['sub'][0], i['sub'][1],
                                        i['levels'], i['df']] for i in info], np.float64)
        print('mosaic', tag, img.shape, len(info), float(np.abs(img).max()))
    # patch histories of one patch: with the shared range profiles and without
    c = origin + (32.0 + 8.0) * 0.5 * np.array(e1) + (32.0 + 8.0) * 0.5 * np.array(e2)
    g = np.linspace(-40.0, 39.0, 9) * 0.5
    pts = c + g[:, None, None] * np.array(e1) + g[None, :, None] * np.array(e2)
    pts = pts.reshape(-1, 3)
    lo, hi = 10, len(ant) - 12
    prof = patches.range_profiles(fx)
    for tag, pr in (('prof', prof), ('direct', None)):
        Sp, a, f0, df2 = patches.patch_history(fx, ant, c, pts, lo, hi, prof=pr)
        rec[f'ph_{tag}_S'] = Sp.astype(np.complex128)
        rec[f'ph_{tag}_geo'] = np.array([f0, df2])
        rec[f'ph_{tag}_a'] = a
    rec['ph_center'], rec['ph_pts'], rec['ph_span'] = c, pts, np.array([lo, hi])
    rec['ph_gate'] = np.array(patches.gate_bins(fx, ant, c, pts, lo, hi))
    pad = patches._padding(fx)
    rec['padding'] = np.array([pad[0], pad[2], pad[3], pad[4]])
    # host helpers
    rec['tile_plan'] = np.array([v for t in [patches.tile_plan(ant - c, col.fmin + col.K * col.df, 80, 80, 0.5, 0.5,
                                                               e1, e2, -40.0)] for v in (t[0], t[1][0], t[1][1], t[2])])
    rec['tile_plan_hard'] = np.array([v for t in [patches.tile_plan(ant - c, col.fmin + col.K * col.df, 400, 80, 0.25,
                                                                    0.5, e1, e2, -70.0)]
                                      for v in (t[0], t[1][0], t[1][1], t[2])])
    rec['levels'] = np.array([patches._levels(n, T, longest=l) for n, T, l in
                              ((80, 32, None), (80, 16, None), (300, 16, 900), (64, 32, 832), (5, 32, None))])
    rec['beam_span'] = np.array(patches.beam_span(beam, len(ant), pts, 1.0))
    gap = np.delete(ant, [5, 6, 40], axis=0)
    fa, fi = patches.fill_gaps(gap)
    rec['gaps_in'], rec['gaps_out'], rec['gaps_idx'] = gap, fa, fi
    counts = [300, 310, 512, 700, 701, 1200, 1210, 1300, 257, 4000]
    rec['buckets_counts'] = np.array(counts)
    rec['buckets_3'] = np.array(patches.choose_buckets(counts, 3.0))
    rec['buckets_0'] = np.array(patches.choose_buckets(counts, 0.0))
    rec['buckets_50'] = np.array(patches.choose_buckets(counts, 50.0, step=64))
    from fastsar import stripmap as sm
    t = np.linspace(-1.2, 1.2, 25)
    for tag, spec in (('taylor', 'taylor'), ('taylor30', ('taylor', 30.0, 5)), ('hann', 'hann'), ('kaiser', 'kaiser'),
                      ('kaiser4', ('kaiser', 4.0)), ('none', None)):
        rec[f'win_{tag}'] = sm.window(spec)(t)
    np.savez_compressed(os.path.join(HERE, 'mosaic.npz'), **rec)
    print('mosaic done', rec['ph_gate'], rec['tile_plan'], rec['beam_span'], rec['buckets_3'])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('FASTSAR_REFERENCE'))
    ap.add_argument('--only', choices=('exact', 'gate', 'weights', 'stack', 'mosaic'), default=None)
    args = ap.parse_args()
    if not args.ref:
        sys.exit('make_golden: name the reference checkout by --ref PATH or FASTSAR_REFERENCE')
    fs = import_reference(args.ref)
    if args.only == 'stack':
        stack(fs)
        return
    if args.only == 'mosaic':
        mosaic(fs)
        return
    if args.only == 'weights':
        weights(fs)
        return
    if args.only == 'exact':
        from fastsar import sim
        from fastsar.exact import ExactFormer
        exact_setup(sim, ExactFormer)
        return
    if args.only == 'gate':
        gate(fs)
        return
    from fastsar import sim, ffbp2, ffbp_cpu, bp
    from fastsar.api import ImageFormer, _window
    from fastsar.exact import ExactFormer
    from fastsar_b200 import sim as mysim

    out = {}
    # --- plans ------------------------------------------------------------------------------------------------
    cases = {}
    c_small = sim.make_collect(res=0.5, scene=60.0, r0=5e3)
    cases['small2'] = (c_small, 128, 128, 0.5, 0.5, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), 16, 2)
    cases['small3'] = (c_small, 128, 128, 0.5, 0.5, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), 16, 3)
    c_600 = sim.make_collect(res=0.5, scene=60.0, r0=600e3)
    cases['orbit3'] = (c_600, 100, 120, 0.5, 0.5, (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), 32, 3)
    w512 = mysim.workload('spotlight_512')
    cases['spot512'] = (w512['col'], 512, 512, 0.25, 0.25, w512['e1'], w512['e2'], 32, 3)
    w12 = mysim.workload('spotlight_12k')
    cases['spot12k'] = (w12['col'], 12288, 8832, 0.2, 0.2, w12['e1'], w12['e2'], 32, 3)
    w4 = mysim.workload('spotlight_4k')
    cases['spot4k'] = (w4['col'], 2048, 2048, 0.25, 0.25, w4['e1'], w4['e2'], 32, 3)
    # patches of uneven sides from one collection (batched workloads), and a 4-level plan
    wp = mysim.spotlight(4096, 2048, 9.6e9, 600e6, 500e3, 50.0, 2.0)
    cases['patch_256x1000'] = (wp, 256, 1000, 0.3, 0.3, (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), 32, 3)
    cases['patch_1500x700'] = (wp, 1500, 700, 0.3, 0.3, (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), 32, 3)
    cases['four_levels'] = (c_small, 256, 256, 0.25, 0.25, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), 16, 4)
    for name, (col, nx, ny, spx, spy, e1, e2, T, nlev) in cases.items():
        _, _, rec = plan_record(ffbp2, col, nx, ny, spx, spy, e1, e2, T, nlev)
        np.savez_compressed(os.path.join(HERE, f'plan_{name}.npz'), **rec)
        print('plan', name, rec['top'], [tuple(rec[f'lv{i}_ints'][:9]) for i in range(int(rec['nlevels']))])
    # choose_splits beyond three levels of factors up to 8 (the fallback to larger factors)
    def splits_or_none(n, T, nl):
        try:
            return ffbp2.choose_splits(n, T, nl)
        except ValueError:
            return ()                                               # the reference refuses: too few levels
    sp = [(n, T, nl, splits_or_none(n, T, nl)) for n, T, nl in
          [(128, 16, 2), (8832, 32, 3), (12288, 32, 3), (100000, 32, 3), (70000, 16, 3), (60000, 16, 3), (300, 32, 1),
           (33, 32, 2), (5000, 16, 2), (12207, 32, 3), (8808, 32, 3), (1000, 32, 1), (4000, 16, 2)]]
    np.savez_compressed(os.path.join(HERE, 'splits.npz'),
                        rows=np.array([[n, T, nl, len(s)] + list(s) + [0] * (3 - len(s)) for n, T, nl, s in sp], np.int64))

    # --- FIR kernels ------------------------------------------------------------------------------------------
    fir = {}
    k = 0
    for n_in, D, pf in [(8192, 3, 0.5), (1647, 8, 0.3), (214, 2, 0.95), (4096, 7, 0.82), (16384, 10, 0.11),
                        (400, 5, 0.67), (1024, 4, 0.25), (512, 2, 0.42)]:
        fr, m = ffbp2.decimator_fir(n_in, D, pf)
        fir[f'k{k}_args'] = np.array([n_in, D, pf])
        fir[f'k{k}_ints'] = np.array([fr['L'], fr['pl'], fr['pr'], fr['n_out'], m])
        fir[f'k{k}_kern'] = np.asarray(fr['kern'])
        k += 1
    np.savez_compressed(os.path.join(HERE, 'fir.npz'), n=np.array(k), **fir)

    # --- the reference's C++ kernels on seeded inputs ----------------------------------------------------------
    L = ffbp_cpu.lib()
    rng = np.random.default_rng(11)
    kr = {}
    Np, P, K, Cn, Dk, Ko = 2, 9, 61, 5, 3, 0
    fr, _ = ffbp2.decimator_fir(K, Dk, 0.6)
    Ko = fr['n_out']
    x = (rng.standard_normal((Np, P, K)) + 1j * rng.standard_normal((Np, P, K))).astype(np.complex64)
    c0 = rng.uniform(-0.5, 0.5, (Np, Cn, P)).astype(np.float32)
    sl = rng.uniform(-0.02, 0.02, (Np, Cn, P)).astype(np.float32)
    taps = np.asarray(fr['kern'], np.float32)
    yre = np.zeros((Np * Cn, P, Ko), np.float32)
    yim = np.zeros((Np * Cn, P, Ko), np.float32)
    L.rot_fir_k_cplx(x.view(np.float32), Np, P, K, c0, sl, Cn, taps, fr['L'], fr['pl'], Dk, Ko, (K - 1) / 2.0, yre, yim)
    kr.update(rk_x=x, rk_c0=c0, rk_sl=sl, rk_taps=taps, rk_ints=np.array([Np, P, K, Cn, fr['L'], fr['pl'], Dk, Ko]),
              rk_yre=yre.copy(), rk_yim=yim.copy())
    xre, xim = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
    L.rot_fir_k(xre, xim, Np, P, K, c0, sl, Cn, taps, fr['L'], fr['pl'], Dk, Ko, (K - 1) / 2.0, yre, yim)
    kr.update(rk2_yre=yre.copy(), rk2_yim=yim.copy())
    B, P2, K2, Dp = 3, 77, 13, 4
    fp, _ = ffbp2.decimator_fir(P2, Dp, 0.5)
    Po = fp['n_out']
    a = rng.standard_normal((B, P2, K2)).astype(np.float32)
    b = rng.standard_normal((B, P2, K2)).astype(np.float32)
    zre = np.zeros((B, Po, K2), np.float32)
    zim = np.zeros((B, Po, K2), np.float32)
    tp = np.asarray(fp['kern'], np.float32)
    L.fir_p(a, b, B, P2, K2, tp, fp['L'], fp['pl'], Dp, Po, zre, zim)
    kr.update(fp_a=a, fp_b=b, fp_taps=tp, fp_ints=np.array([B, P2, K2, fp['L'], fp['pl'], Dp, Po]), fp_zre=zre, fp_zim=zim)
    for T in (16, 32):
        B, Pf, Qf = 3, 7, 11
        d = (rng.standard_normal((B, Pf, Qf)) + 1j * rng.standard_normal((B, Pf, Qf))).astype(np.complex64)
        ux = rng.uniform(-0.9, 0.9, (B, Pf))
        uy = rng.uniform(-0.9, 0.9, (B, Pf))
        dlx = (np.arange(T) - (T - 1) / 2.0) * 0.3
        dly = (np.arange(T) - (T - 1) / 2.0) * 0.45
        a0, a1, fc2 = 64.1, 0.013, 64.4
        ucx, ucy = rng.uniform(-0.5, 0.5, B), rng.uniform(-0.5, 0.5, B)
        rc = rng.uniform(4e3, 6e3, B)
        ore = np.zeros((B, T, T), np.float32)
        oim = np.zeros((B, T, T), np.float32)
        dre, dim = np.ascontiguousarray(d.real), np.ascontiguousarray(d.imag)
        L.final_tiles(dre, dim, B, Pf, Qf, T, ux, uy, dlx, dly, a0, a1, ucx, ucy, rc, fc2, ore, oim, None, None, None)
        w0 = rng.uniform(0.5, 1.5, (B, Pf)).astype(np.float32)
        gx = rng.uniform(-0.01, 0.01, (B, Pf)).astype(np.float32)
        gyr = rng.uniform(-0.01, 0.01, (B, Pf)).astype(np.float32)
        ore_w = np.zeros((B, T, T), np.float32)
        oim_w = np.zeros((B, T, T), np.float32)
        L.final_tiles(dre, dim, B, Pf, Qf, T, ux, uy, dlx, dly, a0, a1, ucx, ucy, rc, fc2, ore_w, oim_w,
                      w0.ctypes.data, gx.ctypes.data, gyr.ctypes.data)
        kr.update({f'ft{T}_d': d, f'ft{T}_ux': ux, f'ft{T}_uy': uy, f'ft{T}_dlx': dlx, f'ft{T}_dly': dly,
                   f'ft{T}_s': np.array([a0, a1, fc2]), f'ft{T}_ucx': ucx, f'ft{T}_ucy': ucy, f'ft{T}_rc': rc,
                   f'ft{T}_out': (ore + 1j * oim).astype(np.complex64), f'ft{T}_w': np.stack([w0, gx, gyr]),
                   f'ft{T}_outw': (ore_w + 1j * oim_w).astype(np.complex64)})
    np.savez_compressed(os.path.join(HERE, 'kernels.npz'), **kr)

    # --- images -----------------------------------------------------------------------------------------------
    rng = np.random.default_rng(1)                                 # the scene of fastsar tests/test_ffbp_cpu.py
    pos = np.stack([rng.uniform(-25, 25, 40), rng.uniform(-25, 25, 40), np.zeros(40)], 1)
    amp = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    S = sim.simulate_brute(c_small, pos, amp).astype(np.complex64)
    rec = dict(S=S, ant=c_small.ant, scal=np.array([c_small.fmin, c_small.df, c_small.K]))
    for nlev in (2, 3):
        f = ImageFormer(c_small.ant, c_small.fmin, c_small.df, c_small.K, 128, 128, 0.5, 0.5, backend='cpu', T=16,
                        levels=nlev)
        rec[f'ffbp_l{nlev}'] = f(S)
    f = ImageFormer(c_small.ant, c_small.fmin, c_small.df, c_small.K, 128, 128, 0.5, 0.5, backend='cpu', T=16,
                    levels=3, window=False)
    rec['ffbp_l3_nowin'] = f(S)
    rec['wp'], rec['wk'] = _window(*S.shape)
    grid = dict(nx=128, ny=128, spx=0.5, spy=0.5, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0))
    rec['exact_cubic'] = ExactFormer(c_small.ant, c_small.fmin, c_small.df, c_small.K, **grid, backend='cpu')(S)
    rec['exact_linear'] = ExactFormer(c_small.ant, c_small.fmin, c_small.df, c_small.K, **grid, backend='cpu',
                                      interp='linear')(S)
    pts = bp.plane_points(**grid)
    rec['bp64'] = bp.backproject(S, c_small.ant, c_small.fmin, c_small.df, pts, backend='cpu', upsample=64)
    np.savez_compressed(os.path.join(HERE, 'image_small.npz'), **rec)
    print('image_small done')

    # the 512-pulse spotlight at 600 km: 32 unit targets plus clutter and noise (seeded; reference simulate_brute)
    rng = np.random.default_rng(2024)
    col = w512['col']
    pos, amp = mysim.scene(rng, 400, 400, 0.25, 0.25, w512['e1'], w512['e2'], n_points=32, clutter_db=-30.0,
                           res=(0.6, 0.5), max_clutter=400)
    S = sim.simulate_brute(col, pos, amp)
    S = mysim.add_noise(S, 10 ** (-40 / 20.0), rng).astype(np.complex64)
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w512['e1'], w512['e2'], backend='cpu')
    img = f(S)
    sub = np.random.default_rng(5).choice(512 * 512, 4096, replace=False)
    pts = bp.plane_points(512, 512, 0.25, 0.25, w512['e1'], w512['e2']).reshape(-1, 3)[sub]
    ref64 = bp.backproject(S, col.ant, col.fmin, col.df, pts, backend='cpu', upsample=64)
    np.savez_compressed(os.path.join(HERE, 'image_spot512.npz'), S=S, ffbp=img, bp64_idx=sub, bp64=ref64,
                        T=np.array(f.T), err=np.array(f.predicted_error_db))
    print('image_spot512 done', f.T, f.predicted_error_db)
    exact_setup(sim, ExactFormer)


if __name__ == '__main__':
    main()
