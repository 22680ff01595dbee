"""Synthetic spotlight collections: geometry, seeded scenes and phase histories.

The phase history follows the CPHD convention of motion compensation to the scene reference point (the origin):
a scatterer of complex amplitude a at x contributes a * exp(-j 4 pi f_k dR / c) to sample k of pulse p, with
dR = |x - ant_p| - |ant_p| (fastsar/sim.py:1-8 states the same convention).

Two geometries are provided:

* `make_collect` -- the broadside linear-track collection the reference's tests use (fastsar/sim.py:45-66): the
  bandwidth, frequency step, aperture length and pulse spacing follow from a resolution, a scene side and a range.
* `spotlight` -- a straight broadside track at a stated slant range, grazing angle and total azimuth aperture, with
  P pulses evenly spaced along track and K frequency samples over a stated bandwidth about the centre frequency
  (df = B / K, fmin = fc - (K // 2) df). This is the geometry of the benchmark workloads.

Phase histories: `simulate_brute` is a direct float64 sum on the host (small cases); `simulate` runs the same sum on
the GPU in float64 through the library (`fastsar_b200._lib`), for the full-size workloads.
"""
from dataclasses import dataclass

import numpy as np

C = 299792458.0


@dataclass
class Collect:
    """One collection: fmin (Hz, sample 0), df (Hz), K samples per pulse, ant [P, 3] antenna phase centres in metres
    about the scene reference point, res the nominal resolution (m). Mirrors fastsar/sim.py:17-42."""
    fmin: float
    df: float
    K: int
    ant: np.ndarray
    res: float

    @property
    def Np(self):
        return self.ant.shape[0]

    @property
    def fref(self):
        """Frequency of sample K // 2."""
        return self.fmin + (self.K // 2) * self.df

    @property
    def freqs(self):
        return self.fmin + self.df * np.arange(self.K)


def _even_ceil(x):
    n = int(np.ceil(x))
    return n + (n & 1)


def make_collect(res=0.3, scene=150.0, r0=10e3, graze_deg=30.0, fc=9.6e9, margin=1.25, offset=(0.0, 0.0, 0.0)):
    """Broadside linear track looking along +x (the reference's test geometry, fastsar/sim.py:45-66).

    The band gives a slant resolution `res`; the frequency step leaves `margin` times the scene diagonal unambiguous
    in range; the aperture gives `res` in azimuth at range r0; the pulse spacing leaves the same extent unambiguous
    in Doppler. Counts are rounded up to even numbers."""
    wavelength = C / fc
    bandwidth = C / (2.0 * res)
    unamb = margin * np.sqrt(2.0) * scene
    df = C / (2.0 * unamb)
    K = _even_ceil(bandwidth / df)
    aperture = r0 * wavelength / (2.0 * res)
    step = wavelength * r0 / (2.0 * unamb)
    P = _even_ceil(aperture / step)
    g = np.deg2rad(graze_deg)
    along = (np.arange(P) - (P - 1) / 2.0) * step
    ant = np.empty((P, 3))
    ant[:, 0] = -r0 * np.cos(g)
    ant[:, 1] = along
    ant[:, 2] = r0 * np.sin(g)
    ant += np.asarray(offset, np.float64)[None, :]
    return Collect(fmin=fc - (K // 2) * df, df=df, K=K, ant=ant, res=res)


def spotlight(P, K, fc, bandwidth, r0, graze_deg, aperture_deg, offset=(0.0, 0.0, 0.0)):
    """Straight broadside track at slant range r0 (m) to the scene centre and grazing angle graze_deg, spanning a total
    azimuth aperture of aperture_deg as seen from the scene centre, with P pulses evenly spaced along track and K
    frequency samples over `bandwidth` Hz centred on fc (df = B / K, fmin = fc - (K // 2) df)."""
    g = np.deg2rad(graze_deg)
    ground = r0 * np.cos(g)
    half = ground * np.tan(0.5 * np.deg2rad(aperture_deg))
    ant = np.empty((P, 3))
    ant[:, 0] = -ground
    ant[:, 1] = np.linspace(-half, half, P)
    ant[:, 2] = r0 * np.sin(g)
    ant += np.asarray(offset, np.float64)[None, :]
    df = bandwidth / K
    res = C / (2.0 * bandwidth)
    return Collect(fmin=fc - (K // 2) * df, df=df, K=K, ant=ant, res=res)


def delta_range(ant, pos):
    """dR [P, N] float64: |pos_n - ant_p| - |ant_p|."""
    d = pos[None, :, :] - ant[:, None, :]
    return np.sqrt((d * d).sum(-1)) - np.linalg.norm(ant, axis=1)[:, None]


def unambiguous_mask(col, pos, guard=20.0):
    """True for scatterers whose range offset stays within c / (4 df) - guard of the reference range on every pulse,
    so that the periodic (in range) phase history holds them without wrapping."""
    lim = C / (4.0 * col.df) - guard
    ok = np.ones(len(pos), bool)
    for p in np.linspace(0, col.Np - 1, min(col.Np, 65)).astype(int):
        ok &= np.abs(delta_range(col.ant[p:p + 1], pos)[0]) < lim
    return ok


def scene(rng, nx, ny, spx, spy, e1=(0.0, 1.0, 0.0), e2=(1.0, 0.0, 0.0), n_points=32, rcs_sigma_db=0.0,
          n_corners=0, corner_db=40.0, clutter_db=None, clutter_per_cell=0.5, res=(1.0, 1.0), max_clutter=200000,
          col=None, fill=0.9):
    """Seeded point-plus-clutter scene on the grid of (nx, ny, spx, spy, e1, e2) -> (pos [N, 3], amp [N] complex).

    Points are uniform over `fill` of the grid; their amplitudes have random phase and, with rcs_sigma_db > 0, a
    log-normal power with that spread in dB (unit median). Corner reflectors sit at +corner_db. Clutter, when
    clutter_db is given, is circular complex Gaussian scatterers, clutter_per_cell per resolution cell (res = the
    two resolutions in metres), scaled so that the clutter power per resolution cell is clutter_db relative to a unit
    target (at most max_clutter scatterers; fewer scatterers carry more power each). With col given, scatterers that
    the collection would alias in range are dropped (unambiguous_mask)."""
    e1, e2 = np.asarray(e1, np.float64), np.asarray(e2, np.float64)
    hx, hy = 0.5 * fill * nx * spx, 0.5 * fill * ny * spy

    def place(n):
        a = rng.uniform(-hx, hx, n)
        b = rng.uniform(-hy, hy, n)
        return a[:, None] * e1[None, :] + b[:, None] * e2[None, :]

    def phase(n):
        return np.exp(2j * np.pi * rng.uniform(0.0, 1.0, n))

    pos = [place(n_points)]
    pw = 10.0 ** (rcs_sigma_db * rng.standard_normal(n_points) / 10.0) if rcs_sigma_db > 0 else np.ones(n_points)
    amp = [np.sqrt(pw) * phase(n_points)]
    if n_corners:
        pos.append(place(n_corners))
        amp.append(10.0 ** (corner_db / 20.0) * phase(n_corners))
    if clutter_db is not None:
        cells = (2 * hx) * (2 * hy) / (res[0] * res[1])
        n = int(min(max_clutter, max(1, round(clutter_per_cell * cells))))
        per = 10.0 ** (clutter_db / 10.0) * cells / n            # power per scatterer
        pos.append(place(n))
        amp.append(np.sqrt(per / 2.0) * (rng.standard_normal(n) + 1j * rng.standard_normal(n)))
    pos, amp = np.concatenate(pos), np.concatenate(amp)
    if col is not None:
        keep = unambiguous_mask(col, pos)
        pos, amp = pos[keep], amp[keep]
    return pos, amp


def simulate_brute(col, pos, amp):
    """Phase history [P, K] complex128 by the direct float64 sum over scatterers, in blocks of scatterers."""
    pos = np.asarray(pos, np.float64)
    amp = np.asarray(amp, np.complex128)
    dr = delta_range(col.ant, pos)                                     # [P, N]
    f = col.freqs
    out = np.zeros((col.Np, col.K), np.complex128)
    nb = max(1, (1 << 22) // max(1, col.Np * col.K))
    for n0 in range(0, len(amp), nb):
        ph = (-4.0 * np.pi / C) * f[None, :, None] * dr[:, None, n0:n0 + nb]
        out += (np.exp(1j * ph) * amp[None, None, n0:n0 + nb]).sum(-1)
    return out


def add_noise(S, sigma, rng):
    """S plus circular complex Gaussian noise of rms `sigma` per sample."""
    return S + (sigma / np.sqrt(2.0)) * (rng.standard_normal(S.shape) + 1j * rng.standard_normal(S.shape))


# ------------------------------------------------------------------------------------------------ benchmark workloads

def workload(name):
    """Collection and grid of a named workload -> dict(col, nx, ny, spx, spy, e1, e2, scene=dict(...)).

    spotlight_512: 512 pulses x 1,024 samples, X band 9.6 GHz, 300 MHz, 600 km, 45 deg grazing, 1.5 deg aperture;
                   512 x 512 pixels at 0.25 m; 32 unit targets in 100 m x 100 m, clutter -30 dB, noise -40 dB.
    spotlight_12k: 16,384 pulses x 8,192 samples, X band 9.6 GHz, 1.2 GHz, 500 km, 55 deg grazing, 3 deg aperture;
                   12,288 x 8,832 pixels at 0.2 m; 2,000 log-normal targets (sigma 10 dB), 10 corners at +40 dB,
                   clutter -25 dB, noise -40 dB; scatterers kept inside the range band the frequency step leaves
                   unambiguous on every pulse.
    spotlight_4k:  4,096 pulses x 4,096 samples at the spotlight_512 geometry (9.6 GHz, 300 MHz, 600 km, 45 deg,
                   1.5 deg) -> 2,048 x 2,048 pixels at 0.25 m."""
    e1, e2 = (0.0, 1.0, 0.0), (1.0, 0.0, 0.0)
    if name == 'spotlight_512':
        col = spotlight(512, 1024, 9.6e9, 300e6, 600e3, 45.0, 1.5)
        return dict(col=col, nx=512, ny=512, spx=0.25, spy=0.25, e1=e1, e2=e2,
                    scene=dict(n_points=32, clutter_db=-30.0, noise_db=-40.0, extent=(100.0, 100.0)))
    if name == 'spotlight_12k':
        col = spotlight(16384, 8192, 9.6e9, 1.2e9, 500e3, 55.0, 3.0)
        return dict(col=col, nx=12288, ny=8832, spx=0.2, spy=0.2, e1=e1, e2=e2,
                    scene=dict(n_points=2000, rcs_sigma_db=10.0, n_corners=10, clutter_db=-25.0, noise_db=-40.0,
                               extent=(2500.0, 1800.0)))
    if name == 'spotlight_4k':
        col = spotlight(4096, 4096, 9.6e9, 300e6, 600e3, 45.0, 1.5)
        return dict(col=col, nx=2048, ny=2048, spx=0.25, spy=0.25, e1=e1, e2=e2,
                    scene=dict(n_points=32, clutter_db=-30.0, noise_db=-40.0, extent=(400.0, 400.0)))
    if name == 'spotlight_12k_strip':
        # the spotlight_12k collection formed to a quarter of its azimuth extent: the same level shapes per parent
        # on about a quarter of the device memory (the profiling case of the level and final kernels)
        w = workload('spotlight_12k')
        w.update(nx=3072, scene=dict(w['scene'], n_points=500, extent=(600.0, 1800.0)))
        return w
    raise ValueError(f'unknown workload {name!r}')


def patch_workload(name='patches_48', seed=0):
    """A batch of uneven image patches from several spotlight collections -> list of dict(col, e1, e2, sp, extent,
    patches=[(ca, cr, na, nr)] (centre along e1 and e2 in metres, pixels along e1 and e2), scene).

    patches_48: 48 patches (8 per collection) with sides drawn log-uniform from 256 to 4,096 pixels (seeded, each side
    held within 80 % of the range and cross-range extents the collection leaves unambiguous), cut from 6 X-band
    spotlight collections of 2,048-16,384 pulses x 2,048-8,192 samples (powers of two), apertures of 1-4 deg,
    bandwidths of 0.6-1.2 GHz, 20-500 km, 35-55 deg grazing; pixel spacing the coarser of the two resolutions (in
    steps of 5 cm); each collection's scene 2,000 log-normal targets (sigma 10 dB) and 10 corners at +40 dB over
    -25 dB clutter across its patches' extent, noise -40 dB."""
    if name != 'patches_48':
        raise ValueError(f'unknown patch workload {name!r}')
    rng = np.random.default_rng(1000 + seed)
    out = []
    for ci in range(6):
        P = int(2 ** rng.integers(11, 15))
        K = int(2 ** rng.integers(11, 14))
        ap = float(rng.uniform(1.0, 4.0))
        bw = float(rng.uniform(0.6e9, 1.2e9))
        r0 = float(rng.choice([20e3, 100e3, 500e3]))
        graze = float(rng.uniform(35.0, 55.0))
        col = spotlight(P, K, 9.6e9, bw, r0, graze, ap)
        res_r = C / (2.0 * bw) / np.cos(np.deg2rad(graze))
        lam = C / 9.6e9
        res_a = lam / (2.0 * np.deg2rad(ap))
        sp = float(np.ceil(max(res_r, res_a) / 0.05) * 0.05)
        swath_r = K * (C / (2.0 * bw)) / np.cos(np.deg2rad(graze))      # unambiguous ground range
        swath_a = lam / (2.0 * np.deg2rad(ap) / P)                        # unambiguous cross range
        lim_r, lim_a = int(0.8 * swath_r / sp), int(0.8 * swath_a / sp)
        ext_r, ext_a = 0.8 * swath_r, 0.8 * swath_a
        patches = []
        for _ in range(8):
            na = int(min(lim_a, np.exp(rng.uniform(np.log(256), np.log(4096)))))
            nr = int(min(lim_r, np.exp(rng.uniform(np.log(256), np.log(4096)))))
            ca = float(rng.uniform(-0.5, 0.5) * max(0.0, ext_a - na * sp))
            cr = float(rng.uniform(-0.5, 0.5) * max(0.0, ext_r - nr * sp))
            patches.append((ca, cr, na, nr))
        out.append(dict(col=col, e1=(0.0, 1.0, 0.0), e2=(1.0, 0.0, 0.0), sp=sp, extent=(ext_a, ext_r),
                        patches=patches, scene=dict(n_points=2000, rcs_sigma_db=10.0, n_corners=10,
                                                    clutter_db=-25.0, noise_db=-40.0)))
    return out


def stack_workload(name='stack_8', seed=0):
    """A repeat-pass stack: passes of one scene on a common grid -> dict(passes=[Collect], offsets [n, 3], nx, ny,
    spx, spy, e1, e2, scene).

    stack_8: 8 wide-angle Ku-band spotlight collections (16 GHz, 800 MHz, 6 deg aperture, 50 km, 45 deg grazing,
    32,768 pulses x 4,096 samples each), the tracks offset from a nominal one by seeded baselines of up to +-50 m
    across track (in height and ground range), each formed to 8,192 x 8,192 pixels at 0.15 m on the grid about the
    common scene origin; the scene 2,000 log-normal targets (sigma 10 dB) and 10 corners at +40 dB over -25 dB
    clutter, noise -40 dB, scatterers kept inside the range band every pass leaves unambiguous."""
    if name != 'stack_8':
        raise ValueError(f'unknown stack workload {name!r}')
    rng = np.random.default_rng(2000 + seed)
    base = spotlight(32768, 4096, 16e9, 800e6, 50e3, 45.0, 6.0)
    offsets = np.zeros((8, 3))
    offsets[1:, 0] = rng.uniform(-50.0, 50.0, 7) / np.sqrt(2.0)
    offsets[1:, 2] = rng.uniform(-50.0, 50.0, 7) / np.sqrt(2.0)
    passes = [Collect(fmin=base.fmin, df=base.df, K=base.K, ant=base.ant + o[None, :], res=base.res) for o in offsets]
    return dict(passes=passes, offsets=offsets, nx=8192, ny=8192, spx=0.15, spy=0.15, e1=(0.0, 1.0, 0.0),
                e2=(1.0, 0.0, 0.0), scene=dict(n_points=2000, rcs_sigma_db=10.0, n_corners=10, clutter_db=-25.0,
                                               noise_db=-40.0))


def simulate(col, pos, amp, out=None, device=None, chunk=65536):
    """Phase history [P, K] complex64 on the GPU (a torch tensor) by the direct sum over scatterers, float64 ranges
    and phases, through ffbp_simulate (fastsar/sim.py:69-90 computes the same sum with a NUFFT). out: a tensor to add
    into (default zeros)."""
    import torch
    from . import _lib
    L = _lib.load()
    dev = device if isinstance(device, torch.device) else torch.device('cuda', torch.cuda.current_device() if device is None else device)
    P, K = col.Np, col.K
    if out is None:
        out = torch.zeros((P, K), dtype=torch.complex64, device=dev)
    ant = torch.from_numpy(np.ascontiguousarray(col.ant, np.float64)).to(dev)
    pos = np.ascontiguousarray(pos, np.float64)
    amp = np.ascontiguousarray(amp, np.complex128)
    s = torch.cuda.current_stream(dev).cuda_stream
    for n0 in range(0, len(amp), chunk):
        p_ = torch.from_numpy(pos[n0:n0 + chunk]).to(dev)
        a_ = torch.from_numpy(amp[n0:n0 + chunk]).to(dev)
        _lib.check(L.ffbp_simulate(ant.data_ptr(), P, K, float(col.fmin), float(col.df), p_.data_ptr(), a_.data_ptr(),
                                   len(a_), out.data_ptr(), s), 'ffbp_simulate')
    return out


def synthetic_history(name, seed=0, device=None, n_clutter=None):
    """The seeded synthetic history of a named workload (workload()) on the GPU: its scene simulated by `simulate`,
    plus complex Gaussian noise at the stated level per sample relative to a unit target. -> (workload dict, S)."""
    import torch
    w = workload(name)
    col, sc = w['col'], w['scene']
    rng = np.random.default_rng(seed)
    ex, ey = sc['extent']
    res = (C / (2.0 * (col.K * col.df)), C / (2.0 * (col.fmin + col.K / 2 * col.df)) /
           (2.0 * np.arctan(0.5 * np.ptp(col.ant[:, 1]) / np.abs(col.ant[0, 0]))))
    kw = dict(n_points=sc['n_points'], rcs_sigma_db=sc.get('rcs_sigma_db', 0.0), n_corners=sc.get('n_corners', 0),
              clutter_db=sc.get('clutter_db'), res=res, col=col, fill=1.0)
    if n_clutter is not None:
        kw['max_clutter'] = n_clutter
    pos, amp = scene(rng, ex / w['spx'], ey / w['spy'], w['spx'], w['spy'], w['e1'], w['e2'], **kw)
    dev = device if isinstance(device, torch.device) else torch.device('cuda', torch.cuda.current_device() if device is None else device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    sigma = 10.0 ** (sc['noise_db'] / 20.0)
    S = (torch.randn((col.Np, col.K, 2), device=dev, generator=g, dtype=torch.float32) * (sigma / np.sqrt(2.0)))
    S = torch.view_as_complex(S).contiguous()
    simulate(col, pos, amp, out=S, device=dev)
    w = dict(w, n_scatterers=len(amp))
    return w, S
