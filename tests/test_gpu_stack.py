"""The stack products on the GPU (fastsar_b200/stack.py, fastsar_b200/products.py, csrc/products.cu) against the
reference's own outputs (tests/golden/stack.npz) and the oracle (oracle/stack_oracle.py) on seeded images, and
size-independent properties at the 8,192 x 8,192 grid of the repeat-pass stack."""
import os

import numpy as np
import pytest

import stack_oracle as so   # oracle/ is on the path (conftest.py)

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def g():
    return dict(np.load(os.path.join(HERE, 'golden', 'stack.npz')))


@pytest.fixture(scope='module')
def mods():
    import torch
    from fastsar_b200 import stack, products, _lib
    _lib.load()
    return torch, stack, products


def _cuda(torch, x):
    return torch.as_tensor(x).cuda()


def test_box_means_bitwise(g, mods):
    torch, st, _ = mods
    assert np.array_equal(st.intensity_box(_cuda(torch, g['a']), 5).cpu().numpy(), g['box5_a'])
    assert np.array_equal(st.intensity_box(_cuda(torch, g['c']), 4).cpu().numpy(), g['box4_c'])
    # a real image: its square, and a float taken as it is
    amp = np.abs(g['b']).astype(np.float32)
    assert np.array_equal(st.intensity_box(_cuda(torch, amp), 7).cpu().numpy(), so.box(so.power(amp), 7))
    p = so.power(g['a'])
    out = st.intensity_box(_cuda(torch, p), 9, kind=0).cpu().numpy()
    assert np.array_equal(out, so.box(p, 9))


def test_detected(g, mods):
    torch, st, _ = mods
    for img, w, key in ((g['a'], 5, 'det_a'), (g['b'], 5, 'det_b'), (g['c'], 3, 'det3_c')):
        np.testing.assert_allclose(st.detected(img, w).cpu().numpy(), g[key], rtol=0, atol=2e-4)


@pytest.mark.parametrize('tag,hp', [('hp', 32.0), ('nohp', None)])
def test_peak_and_estimate_match_reference(g, mods, tag, hp):
    torch, st, _ = mods
    da, db = _cuda(torch, g['det_a']), _cuda(torch, g['det_b'])
    d, z, rho, clear = st.peak(da, db, 16, highpass=hp)
    ref = g[f'peak_{tag}']
    np.testing.assert_allclose(d, ref[:2], atol=2e-4)
    np.testing.assert_allclose([z, rho], ref[2:4], rtol=2e-4)
    assert float(clear) == ref[4]
    e = st.estimate(da, db, 0.25, 0.3, 16, 2, hp)
    np.testing.assert_allclose(e['shift_px'], g[f'est_{tag}_shift_px'], atol=2e-4)
    assert e['found'] == bool(g[f'est_{tag}_found'])
    assert e['tiles'] == int(g[f'est_{tag}_tiles']) and e['tiles_used'] == int(g[f'est_{tag}_tiles_used'])
    np.testing.assert_array_equal(e['tile_used'], g[f'est_{tag}_tile_used'])
    np.testing.assert_allclose(e['tile_residuals'], g[f'est_{tag}_tile_residuals'], atol=2e-4)
    np.testing.assert_allclose(e['tile_significance'], g[f'est_{tag}_tile_significance'], rtol=2e-4)


def test_peak_about_a_translation(g, mods):
    torch, st, _ = mods
    d, z, rho, clear = st.peak(_cuda(torch, g['det_a'][:64, :80]), _cuda(torch, g['det_b'][:64, :80]), 16,
                               around=(-3, 3), narrow=8)
    ref = g['peak_tile']
    np.testing.assert_allclose(d, ref[:2], atol=2e-4)
    np.testing.assert_allclose([z, rho], ref[2:4], rtol=2e-4)
    assert float(clear) == ref[4]


def test_translate_matches_reference(g, mods):
    torch, st, _ = mods
    out = st.translate(_cuda(torch, so.power(g['b'])), (1.3, -0.4)).cpu().numpy()
    np.testing.assert_allclose(out, g['tr_real'], rtol=0, atol=2e-6 * float(np.abs(g['tr_real']).max()))
    for d, key in (((2.25, -1.5), 'tr_cplx'), ((-3.0, 2.0), 'tr_whole')):
        out = st.translate(_cuda(torch, g['c']), d).cpu().numpy()
        np.testing.assert_array_equal(out == 0, g[key] == 0)
        np.testing.assert_allclose(out, g[key], rtol=0, atol=2e-6 * float(np.abs(g[key]).max()))
    # whole pixels only: the array moved, bit for bit
    assert np.array_equal(st.translate(_cuda(torch, g['c']), (-3.0, 2.0)).cpu().numpy(), g['tr_whole'])


@pytest.mark.parametrize('tag,eq,imgs', [('small', None, 'abc'), ('plain', None, 'm'), ('mean', 'mean', 'm'),
                                         ('median', 'median', 'm')])
def test_mean_matches_reference(g, mods, tag, eq, imgs):
    torch, st, _ = mods
    images = (g['a'], g['b'], g['c']) if imgs == 'abc' else (g['m_a'], g['m_b'], g['m_c'])
    acc = st.Mean(eq, 32)
    for img, w in zip(images, g[f'mean_{tag}_weights']):
        acc.add(dict(image=img), float(w))
    M = acc.image()
    np.testing.assert_allclose(acc.gains, g[f'mean_{tag}_gains'], rtol=1e-6)
    if eq is None:     # the reference's float32 products and sums, bit for bit
        assert np.array_equal(M.cpu().numpy(), g[f'mean_{tag}_M'])
    else:
        np.testing.assert_allclose(M.cpu().numpy(), g[f'mean_{tag}_M'], rtol=2e-6, atol=0)
    L = acc.looks(M)
    if np.isnan(g[f'mean_{tag}_looks']):
        assert L['looks'] is None
        return
    for k in ('looks', 'looks_single', 'looks_by_n', 'looks_ideal', 'looks_independent', 'brightness_spread_db'):
        np.testing.assert_allclose(L[k], g[f'mean_{tag}_{k}'], rtol=1e-4)
    assert L['tiles_selected'] == int(g[f'mean_{tag}_tiles_selected'])
    np.testing.assert_array_equal(L['homogeneous'], g[f'mean_{tag}_homogeneous'])


def test_mean_product(g, mods):
    torch, st, _ = mods
    prods = [dict(image=g['m_a'], spx=0.15, spy=0.15, name='a'), dict(image=g['m_b'], spx=0.15, spy=0.15),
             dict(image=g['m_c'], spx=0.15, spy=0.15)]
    res = st.mean(prods, weights=[1.0, 2.0, 0.5])
    assert isinstance(res['image'], np.ndarray) and res['count'] == 3 and res['name'] == 'a'
    np.testing.assert_allclose(res['image'], np.sqrt(g['mean_plain_M']), rtol=2e-7)
    np.testing.assert_allclose(res['looks'], g['mean_plain_looks'], rtol=1e-4)
    with pytest.raises(ValueError, match='grid'):
        st.mean([prods[0], dict(image=g['a'], spx=0.15, spy=0.15)])
    with pytest.raises(ValueError, match='positive'):
        st.mean(prods, weights=[1.0, 0.0, 1.0])


def test_pair_products_match_reference(g, mods):
    torch, st, pr = mods
    np.testing.assert_allclose(pr.multilook(g['a'], 2, 3), g['ml_a_2_3'], rtol=2e-6)
    np.testing.assert_allclose(pr.interferogram(g['a'], g['b'], 2, 2), g['ifg_ab_2_2'], rtol=0,
                               atol=2e-6 * float(np.abs(g['ifg_ab_2_2']).max()))
    for (x, y, w1, w2), key in (((g['a'], g['b'], 5, 5), 'coh_ab_5_5'), ((g['a'], g['c'], 7, 3), 'coh_ac_7_3'),
                                ((g['a'], g['b'], 4, 6), 'coh_ab_4_6')):
        np.testing.assert_allclose(pr.coherence(x, y, w1, w2), g[key], rtol=0, atol=2e-6)


def test_register_translates_detected_images(mods):
    """register on amplitude images against the oracle's estimate and translation of the same images."""
    torch, st, _ = mods
    rng = np.random.default_rng(7)
    n1, n2 = 384, 448
    k1, k2 = np.fft.fftfreq(n1)[:, None], np.fft.fftfreq(n2)[None, :]
    F = np.fft.fft2(rng.standard_normal((n1, n2)) + 1j * rng.standard_normal((n1, n2)))
    band = (np.abs(k1) < 0.3) & (np.abs(k2) < 0.3)
    a = np.fft.ifft2(F * band).astype(np.complex64)
    b = np.fft.ifft2(F * band * np.exp(2j * np.pi * (k1 * 5.4 + k2 * -7.7))).astype(np.complex64)
    A, B = np.abs(a).astype(np.float32), np.abs(b).astype(np.float32)
    prods = [dict(image=A, spx=0.2, spy=0.25), dict(image=B, spx=0.2, spy=0.25)]
    out = st.register(prods, max_shift=32, tiles=4)
    est = out[1]['registration']
    ref = so.estimate(so.detected(A, 5), so.detected(B, 5), 0.2, 0.25, 32, 4, 32.0)
    assert est['found'] and ref['found']
    np.testing.assert_allclose(est['shift_px'], ref['shift_px'], atol=1e-3)
    np.testing.assert_allclose(est['shift_px'], (-5.4, 7.7), atol=0.1)
    assert est['tiles_used'] == ref['tiles_used']
    np.testing.assert_allclose(out[1]['shift'], est['shift'])
    want = so.translate(B, est['shift_px'])
    np.testing.assert_allclose(out[1]['image'], want, rtol=0, atol=2e-6 * float(want.max()))
    assert out[0]['registration']['reference']
    # complex images: estimated, not translated
    cx = st.register([dict(image=a, spx=0.2, spy=0.25), dict(image=b, spx=0.2, spy=0.25)], max_shift=32, tiles=4)
    assert cx[1]['registration']['found'] and cx[1]['image'] is b and 'not translated' in cx[1]['notes'][-1]
    with pytest.raises(ValueError, match='reform'):
        st.register(prods, apply='reform')


# ------------------------------------------------------------------------------------------------ full grid
def _speckle(torch, n, seed, band=0.35):
    """A seeded complex speckle image n x n on the device, band-limited to `band` of the sampling rate."""
    gen = torch.Generator(device='cuda').manual_seed(seed)
    w = torch.randn((n, n), dtype=torch.complex64, device='cuda', generator=gen)
    F = torch.fft.fft2(w)
    k = torch.fft.fftfreq(n, device='cuda').abs() < band
    return torch.fft.ifft2(F * (k[:, None] & k[None, :])).contiguous()


def test_full_grid_properties(mods):
    """At the stack's 8,192 x 8,192 grid: coherence of an image with a complex multiple of itself is 1, the mean of
    equal images is their intensity bit for bit, a whole-pixel translation moves the array bit for bit, and a known
    sub-pixel translation is recovered by the registration."""
    torch, st, pr = mods
    n = 8192
    a = _speckle(torch, n, 11)
    coh = pr.coherence(a, a * (0.3 - 0.7j), 7, 7)
    assert float((coh - 1).abs().max()) < 2e-6
    acc = st.Mean(None, 32)
    for _ in range(4):                    # 4 p / 4 = p exactly
        acc.add(dict(image=a), 1.0)
    p = st.intensity_box(a, 1)
    assert torch.equal(acc.image(), p)
    moved = st.translate(p, (5.0, -3.0))
    assert torch.equal(moved[:-5, 3:], p[5:, :-3]) and not moved[-5:].any() and not moved[:, :3].any()
    # a whole-pixel displacement is found to a few hundredths; a fractional one to the detected images' precision
    # on speckle (the reference's own case, stack.npz: -3.23, 2.64 for -3.3, 2.6)
    da = st.detected(a, 5)
    for d, tol in (((3.0, -2.0), 0.02), ((2.3, -1.6), 0.1)):
        f1, f2 = torch.fft.fftfreq(n, device='cuda')[:, None], torch.fft.fftfreq(n, device='cuda')[None, :]
        b = torch.fft.ifft2(torch.fft.fft2(a) * torch.exp(2j * np.pi * (f1 * d[0] + f2 * d[1]))).contiguous()
        e = st.estimate(da, st.detected(b, 5), 0.15, 0.15, 16, 4)
        assert e['found'] and e['tiles_used'] == 16
        np.testing.assert_allclose(e['shift_px'], (-d[0], -d[1]), atol=tol)
        del b
