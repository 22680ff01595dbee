"""The stack products' oracle (oracle/stack_oracle.py) against the reference's own outputs (tests/golden/stack.npz,
made by tests/golden/make_golden.py --only stack from fastsar/stack.py and fastsar/products.py)."""
import os

import numpy as np
import pytest

import stack_oracle as so   # oracle/ is on the path (conftest.py)

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def g():
    return dict(np.load(os.path.join(HERE, 'golden', 'stack.npz')))


def test_box_bitwise(g):
    assert np.array_equal(so.box(so.power(g['a']), 5), g['box5_a'])
    assert np.array_equal(so.box(so.power(g['c']), 4), g['box4_c'])


def test_detected(g):
    for img, w, key in ((g['a'], 5, 'det_a'), (g['b'], 5, 'det_b'), (g['c'], 3, 'det3_c')):
        np.testing.assert_allclose(so.detected(img, w), g[key], rtol=0, atol=1e-4)


@pytest.mark.parametrize('tag,hp', [('hp', 32.0), ('nohp', None)])
def test_peak_and_estimate(g, tag, hp):
    d, z, rho, clear = so.peak(g['det_a'], g['det_b'], 16, highpass=hp)
    ref = g[f'peak_{tag}']
    np.testing.assert_allclose(d, ref[:2], atol=1e-6)
    np.testing.assert_allclose([z, rho], ref[2:4], rtol=1e-5)
    assert float(clear) == ref[4]
    e = so.estimate(g['det_a'], g['det_b'], 0.25, 0.3, 16, 2, hp)
    np.testing.assert_allclose(e['shift_px'], g[f'est_{tag}_shift_px'], atol=1e-6)
    np.testing.assert_allclose(e['shift'], g[f'est_{tag}_shift'], atol=1e-6)
    assert e['found'] == bool(g[f'est_{tag}_found'])
    assert e['tiles'] == int(g[f'est_{tag}_tiles']) and e['tiles_used'] == int(g[f'est_{tag}_tiles_used'])
    np.testing.assert_array_equal(e['tile_used'], g[f'est_{tag}_tile_used'])
    np.testing.assert_allclose(e['tile_residuals'], g[f'est_{tag}_tile_residuals'], atol=1e-6)
    np.testing.assert_allclose(e['tile_significance'], g[f'est_{tag}_tile_significance'], rtol=1e-5)
    for k in ('significance', 'correlation', 'residual_rms', 'residual_median', 'residual_worst'):
        np.testing.assert_allclose(e[k], g[f'est_{tag}_{k}'], rtol=1e-5, atol=1e-9)


def test_peak_about_a_translation(g):
    d, z, rho, clear = so.peak(g['det_a'][:64, :80], g['det_b'][:64, :80], 16, around=(-3, 3), narrow=8)
    ref = g['peak_tile']
    np.testing.assert_allclose(d, ref[:2], atol=1e-6)
    np.testing.assert_allclose([z, rho], ref[2:4], rtol=1e-5)
    assert float(clear) == ref[4]


def test_translate(g):
    scale = float(np.abs(g['tr_real']).max())
    np.testing.assert_allclose(so.translate(so.power(g['b']), (1.3, -0.4)), g['tr_real'], rtol=0, atol=1e-6 * scale)
    for d, key in (((2.25, -1.5), 'tr_cplx'), ((-3.0, 2.0), 'tr_whole')):
        out = so.translate(g['c'], d)
        assert out.dtype == g[key].dtype
        np.testing.assert_array_equal(out == 0, g[key] == 0)
        np.testing.assert_allclose(out, g[key], rtol=0, atol=1e-6 * float(np.abs(g[key]).max()))


@pytest.mark.parametrize('tag,eq,imgs', [('small', None, 'abc'), ('plain', None, 'm'), ('mean', 'mean', 'm'),
                                         ('median', 'median', 'm')])
def test_mean(g, tag, eq, imgs):
    images = (g['a'], g['b'], g['c']) if imgs == 'abc' else (g['m_a'], g['m_b'], g['m_c'])
    acc = so.Mean(eq, 32)
    for img, w in zip(images, g[f'mean_{tag}_weights']):
        acc.add(img, float(w))
    M = acc.image()
    np.testing.assert_allclose(acc.gains, g[f'mean_{tag}_gains'], rtol=1e-6)
    np.testing.assert_allclose(M, g[f'mean_{tag}_M'], rtol=1e-6, atol=0)
    L = acc.looks(M)
    if np.isnan(g[f'mean_{tag}_looks']):
        assert L['looks'] is None
        return
    for k in ('looks', 'looks_single', 'looks_by_n', 'looks_ideal', 'looks_independent', 'brightness_spread_db'):
        np.testing.assert_allclose(L[k], g[f'mean_{tag}_{k}'], rtol=1e-5)
    assert L['tiles_selected'] == int(g[f'mean_{tag}_tiles_selected'])
    np.testing.assert_array_equal(L['homogeneous'], g[f'mean_{tag}_homogeneous'])


def test_level(g):
    p = so.power(g['c'])
    np.testing.assert_allclose(so.level(p, 'mean'), g['level_mean'], rtol=1e-6)
    np.testing.assert_allclose(so.level(p, 'median'), g['level_median'], rtol=1e-6)


def test_pair_products(g):
    np.testing.assert_allclose(so.multilook(g['a'], 2, 3), g['ml_a_2_3'], rtol=1e-6)
    np.testing.assert_allclose(so.interferogram(g['a'], g['b'], 2, 2), g['ifg_ab_2_2'], rtol=0,
                               atol=1e-6 * float(np.abs(g['ifg_ab_2_2']).max()))
    for (x, y, w1, w2), key in (((g['a'], g['b'], 5, 5), 'coh_ab_5_5'), ((g['a'], g['c'], 7, 3), 'coh_ac_7_3'),
                                ((g['a'], g['b'], 4, 6), 'coh_ab_4_6')):
        np.testing.assert_allclose(so.coherence(x, y, w1, w2), g[key], rtol=0, atol=1e-12)
