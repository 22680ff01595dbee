"""The planner (fastsar_b200.plan) against the reference planner's own output (tests/golden/plan_*.npz, written by
tests/golden/make_golden.py from fastsar/ffbp2.py): every integer field bit-exact (tile grid, splits, decimations,
filter lengths and offsets, sizes), every float field to 1e-12 relative, the filter kernels and the float64
collection geometry (fastsar tests/test_units.py:90-110 pins decimator_fir the same way)."""
import glob
import os

import numpy as np
import pytest

from fastsar_b200 import plan as P_
from fastsar_b200.sim import Collect

from conftest import GOLDEN

CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, 'plan_*.npz')))


def _close(a, b, rtol=1e-12, atol=1e-9):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = np.abs(b).max() if b.size else 0.0
    np.testing.assert_allclose(a, b, rtol=rtol, atol=max(atol, rtol * scale))


def _stats(a):
    a = np.asarray(a, np.float64).ravel()
    step = max(1, len(a) // 4096)
    return np.concatenate([[len(a), a.sum(), (a * a).sum()], a[::step]])


def _check_array(mine, gold):
    mine = np.asarray(mine, np.float64)
    if mine.shape == gold.shape:
        _close(mine, gold)
    else:                                                    # a large array: its summary
        s = _stats(mine)
        assert s[0] == gold[0]
        _close(s[3:], gold[3:])
        _close(s[1:3], gold[1:3], rtol=1e-9)


def _plan_of(rec):
    fmin, df, K, nx, ny, spx, spy, T, nlev, pmax = rec['scal']
    col = Collect(fmin=fmin, df=df, K=int(K), ant=rec['ant'], res=0.5)
    return col, P_.make_plan(col, int(nx), int(ny), spx, spy, T=int(T), nlev=int(nlev), pmax=pmax, e1=rec['e1'], e2=rec['e2'])


@pytest.mark.parametrize('case', CASES)
def test_plan_matches_reference(golden, case):
    rec = golden('plan_' + case)
    col, plan = _plan_of(rec)
    assert [plan['T'], plan['Nx'], plan['Ny'], plan['ox'], plan['oy']] == rec['top'].tolist()
    assert len(plan['levels']) == int(rec['nlevels'])
    for i, l in enumerate(plan['levels']):
        fk, fp = l['fir_k'], l['fir_p']
        ints = [l['sx'], l['sy'], l['C'], l['Dk'], l['Dp'], l['K'], l['P'], l['Ko'], l['Po'],
                fk['L'] if fk else -1, fk['pl'] if fk else -1, fk['pr'] if fk else -1, fk['n_out'] if fk else -1,
                fp['L'] if fp else -1, fp['pl'] if fp else -1, fp['pr'] if fp else -1, fp['n_out'] if fp else -1]
        assert ints == rec[f'lv{i}_ints'].tolist(), (case, i)
        _close([l['f0'], l['df'], l['pass_k'], l['pass_p'], l['dec_k'][2], l['dec_p'][2]], rec[f'lv{i}_f'])
        if fk:
            _close(fk['kern'], rec[f'lv{i}_kk'], rtol=1e-13)
        if fp:
            _close(fp['kern'], rec[f'lv{i}_kp'], rtol=1e-13)
        for key in ('cen', 'd', 'ref', 'pidx'):
            _check_array(l[key], rec[f'lv{i}_{key}'])
    f = plan['final']
    _close([f['P'], f['K'], f['f0'], f['df'], f['fc']], rec['final_f'])
    _check_array(f['cen'], rec['final_cen'])


@pytest.mark.parametrize('case', CASES)
def test_collection_arrays_match_reference(golden, case):
    rec = golden('plan_' + case)
    col, plan = _plan_of(rec)
    coll = P_.collection_arrays(plan, col.ant)
    for i, c in enumerate(coll['levels']):
        for key in ('u', 'r0', 'c0', 'slope'):
            if f'ca{i}_{key}' in rec:
                g = rec[f'ca{i}_{key}']
                if key in ('c0', 'slope'):
                    a = np.asarray(c[key])
                    assert a.dtype == np.float32
                    if a.shape == g.shape:
                        # float32 of float64 phases: equal, or one float32 ulp apart where the wrap or the rounding of
                        # an ulp-level float64 difference flips
                        d = np.abs(a.astype(np.float64) - g.astype(np.float64))
                        assert (d <= 2 * np.spacing(np.abs(g).astype(np.float32)).astype(np.float64) + 1e-12).mean() > 0.999
                        assert d.max() < 1e-5
                    else:
                        s = _stats(a)
                        assert s[0] == g[0]
                        np.testing.assert_allclose(s[3:], g[3:], atol=1e-5)
                else:
                    _check_array(c[key], g)
    _check_array(coll['final']['u'], rec['caf_u'])
    _check_array(coll['final']['r0'], rec['caf_r0'])


@pytest.mark.parametrize('case', CASES)
def test_choose_T_matches_reference(golden, case):
    rec = golden('plan_' + case)
    fmin, df, K, nx, ny, spx, spy = rec['scal'][:7]
    fmax = fmin + K * df
    T, err = P_.choose_T(rec['ant'], fmax, int(nx), int(ny), spx, spy, rec['e1'], rec['e2'])
    assert T == int(rec['choose_T'][0])
    _close(err, rec['choose_T'][1], rtol=1e-9)
    for t, e in zip((16, 32), rec['phase_err']):
        _close(P_.final_phase_error(rec['ant'], fmax, int(nx), int(ny), spx, spy, rec['e1'], rec['e2'], t), e, rtol=1e-9)


def test_choose_splits_matches_reference(golden):
    for row in golden('splits')['rows']:
        n, T, nl, ns = (int(v) for v in row[:4])
        if ns == 0:
            with pytest.raises(ValueError, match='cannot split'):
                P_.choose_splits(n, T, nl)
        else:
            assert list(P_.choose_splits(n, T, nl)) == row[4:4 + ns].tolist(), (n, T, nl)


def test_decimator_fir_matches_reference(golden):
    g = golden('fir')
    for k in range(int(g['n'])):
        n_in, D, pf = g[f'k{k}_args']
        fr, m = P_.decimator_fir(int(n_in), int(D), pf)
        assert [fr['L'], fr['pl'], fr['pr'], fr['n_out'], m] == g[f'k{k}_ints'].tolist()
        _close(fr['kern'], g[f'k{k}_kern'], rtol=1e-13)
        assert P_.decimator_shape(int(n_in), int(D), pf) == (fr['n_out'], m)


def test_decimator_rows_sum_to_one():
    """Every input sample's weights over the outputs sum to one (the normalisation the kernel carries)."""
    fr, m = P_.decimator_fir(300, 4, 0.5)
    F = np.zeros((300, fr['n_out']))
    for j in range(fr['n_out']):
        for r in range(fr['L']):
            i = 4 * j + r - fr['pl']
            if 0 <= i < 300:
                F[i, j] = fr['kern'][r]
    interior = slice(fr['L'], 300 - fr['L'])
    np.testing.assert_allclose(F.sum(1)[interior], 1.0, atol=1e-12)


def weight_fn(P):
    """The aperture weight of tests/golden/weights.npz (tests/golden/make_golden.py weight_fn): a raised cosine over
    the pulses times a linear ramp over the scene."""
    def w(q, p):
        q, p = np.asarray(q, np.float64), np.asarray(p, np.float64)
        over_p = 0.55 + 0.45 * np.cos(np.pi * (p - 0.5 * (P - 1)) / P)
        over_q = 1.0 + 0.006 * q[:, 0] - 0.004 * q[:, 1]
        return over_p[:, None] * over_q[None, :]
    return w


def test_final_weights_match_reference(golden):
    """plan.final_weights against the reference's api.final_weights (fastsar/api.py:203-244) on the test scene's
    2-level plan: the Gauss-Legendre mean, the centre-pulse form and the gradient form, to float32 rounding."""
    g, img = golden('weights'), golden('image_small')
    fmin, df, K = img['scal']
    col = Collect(fmin=float(fmin), df=float(df), K=int(K), ant=img['ant'], res=0.5)
    plan = P_.make_plan(col, 128, 128, 0.5, 0.5, T=16, nlev=2, pmax=0.4, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0))
    P = img['ant'].shape[0]
    w = weight_fn(P)
    np.testing.assert_allclose(P_.final_weights(plan, w, P), g['w_plain'], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(P_.final_weights(plan, w, P, nodes=1), g['w_centre'], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(P_.final_weights(plan, w, P, grad=True), g['w_grad'], rtol=1e-5, atol=1e-7)


def test_packaged_level_options_cache_is_well_formed(tmp_path, monkeypatch):
    """The packaged tuning cache (fastsar_b200/data/level_opts.json, written by python -m fastsar_b200.tune): every
    key a level signature of 10 integers, every value a dict of ffbp_tc_opts fields with values the launcher takes;
    and a cache written through FASTSAR_TUNE_CACHE reads back the same."""
    import json
    from fastsar_b200 import tune
    doc = json.load(open(tune.PACKAGED_CACHE))
    assert doc['levels']
    for k, v in doc['levels'].items():
        assert len([int(x) for x in k.split(',')]) == 10
        assert set(v) <= {'nt', 'sb', 'copies', 'repeat', 'fir', 'consumers'}
        assert v.get('consumers', 8) in (4, 8, 12)
        assert v.get('copies', 2) in (2, 4) and v.get('fir', 1) in (1, 2) and v.get('repeat', 0) in (0, 1)
        assert v.get('nt', 16) % 16 == 0 and 2 <= v.get('sb', 2) <= 4
    monkeypatch.setattr(tune, '_LEVEL_CACHE', {})
    monkeypatch.setattr(tune, '_CACHE_LOADED', False)
    tune._load_cache()
    assert len(tune._LEVEL_CACHE) == len(doc['levels'])
    path = str(tmp_path / 'cache.json')
    tune._LEVEL_CACHE[(1, 2, 3, 4, 5, 6, 7, 8, 9, 10)] = dict(nt=64, fir=2)
    tune._save_cache(path)
    monkeypatch.setenv('FASTSAR_TUNE_CACHE', path)
    monkeypatch.setattr(tune, '_LEVEL_CACHE', {})
    monkeypatch.setattr(tune, '_CACHE_LOADED', False)
    tune._load_cache()
    assert tune._LEVEL_CACHE[(1, 2, 3, 4, 5, 6, 7, 8, 9, 10)] == dict(nt=64, fir=2)
