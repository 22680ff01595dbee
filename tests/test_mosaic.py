"""The patch mosaic's host side (fastsar_b200/mosaic.py) against the reference's own outputs (tests/golden/mosaic.npz,
made by tests/golden/make_golden.py --only mosaic from fastsar/patches.py and fastsar/stripmap.py): the tile plan,
level counts, beam spans, gap filling, program buckets, frequency padding, range gate and azimuth windows."""
import os

import numpy as np
import pytest

from fastsar_b200 import mosaic as mo

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def g():
    return dict(np.load(os.path.join(HERE, 'golden', 'mosaic.npz')))


def _beam(ant):
    def beam(idx, pts):
        d = np.asarray(pts, np.float64)[None, :, :] - ant[np.asarray(idx)][:, None, :]
        return d[..., 1] / 20.0
    return beam


def _fx(g):
    return dict(S=g['S'], fmin=float(g['fmin']), df=float(g['df']), ref=g['ref'], band=tuple(g['band']))


def test_tile_plan_and_levels(g):
    c, ant = g['ph_center'], g['ant']
    fmax = float(g['fmin']) + g['S'].shape[1] * float(g['df'])
    e1, e2 = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)
    T, s, err = mo.tile_plan(ant - c, fmax, 80, 80, 0.5, 0.5, e1, e2, -40.0)
    np.testing.assert_allclose([T, s[0], s[1], err], g['tile_plan'], rtol=1e-9)
    T, s, err = mo.tile_plan(ant - c, fmax, 400, 80, 0.25, 0.5, e1, e2, -70.0)
    np.testing.assert_allclose([T, s[0], s[1], err], g['tile_plan_hard'], rtol=1e-9)
    got = [mo._levels(n, T, longest=l) for n, T, l in ((80, 32, None), (80, 16, None), (300, 16, 900), (64, 32, 832),
                                                      (5, 32, None))]
    assert got == list(g['levels'])


def test_beam_span_and_gaps(g):
    assert mo.beam_span(_beam(g['ant']), len(g['ant']), g['ph_pts'], 1.0) == tuple(g['beam_span'])
    fa, fi = mo.fill_gaps(g['gaps_in'])
    np.testing.assert_array_equal(fi, g['gaps_idx'])
    np.testing.assert_allclose(fa, g['gaps_out'], rtol=0, atol=1e-9)
    a, i = mo.fill_gaps(g['ant'])
    assert a.shape == g['ant'].shape and np.array_equal(i, np.arange(len(a)))


def test_choose_buckets(g):
    counts = list(g['buckets_counts'])
    assert mo.choose_buckets(counts, 3.0) == list(g['buckets_3'])
    assert mo.choose_buckets(counts, 0.0) == list(g['buckets_0'])
    assert mo.choose_buckets(counts, 50.0, step=64) == list(g['buckets_50'])
    assert mo.choose_buckets([0, -3], 1.0) == []


def test_padding_and_gate(g):
    fx = _fx(g)
    guard, band, npl, K2, f0 = mo._padding(fx)
    np.testing.assert_allclose([guard, npl, K2, f0], g['padding'], rtol=1e-12)
    lo, hi = (int(v) for v in g['ph_span'])
    assert mo.gate_bins(fx, g['ant'], g['ph_center'], g['ph_pts'], lo, hi) == tuple(g['ph_gate'])


@pytest.mark.parametrize('tag,spec', [('taylor', 'taylor'), ('taylor30', ('taylor', 30.0, 5)), ('hann', 'hann'),
                                      ('kaiser', 'kaiser'), ('kaiser4', ('kaiser', 4.0)), ('none', None)])
def test_windows(g, tag, spec):
    t = np.linspace(-1.2, 1.2, 25)
    np.testing.assert_allclose(mo.window(spec)(t), g[f'win_{tag}'], rtol=1e-12, atol=1e-14)
    with pytest.raises(ValueError, match='unknown window'):
        mo.window('boxcar')
