"""The patch mosaic on the GPU (fastsar_b200/mosaic.py, csrc/mosaic.cu) against the reference's own outputs
(tests/golden/mosaic.npz: fastsar/patches.py form_mosaic with its CPU former, and patch_history)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
E1, E2 = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)


@pytest.fixture(scope='module')
def g():
    return dict(np.load(os.path.join(HERE, 'golden', 'mosaic.npz')))


def _fx(g):
    return dict(S=g['S'], fmin=float(g['fmin']), df=float(g['df']), ref=g['ref'], band=tuple(g['band']))


def _beam(ant):
    def beam(idx, pts):
        d = np.asarray(pts, np.float64)[None, :, :] - ant[np.asarray(idx)][:, None, :]
        return d[..., 1] / 20.0
    return beam


def _rel_db(a, b):
    return 10 * np.log10(np.sum(np.abs(a.astype(np.complex128) - b) ** 2) / np.sum(np.abs(b) ** 2))


@pytest.mark.parametrize('tag', ['prof', 'direct'])
def test_patch_history_matches_reference(g, tag):
    from fastsar_b200 import mosaic as mo
    fx = _fx(g)
    lo, hi = (int(v) for v in g['ph_span'])
    prof = mo.range_profiles(fx) if tag == 'prof' else None
    S, a, f0, df2 = mo.patch_history(fx, g['ant'], g['ph_center'], g['ph_pts'], lo, hi, prof=prof)
    ref = g[f'ph_{tag}_S']
    assert tuple(S.shape) == ref.shape
    assert _rel_db(S.cpu().numpy(), ref) < -110
    np.testing.assert_allclose([f0, df2], g[f'ph_{tag}_geo'], rtol=1e-12)
    np.testing.assert_allclose(a, g[f'ph_{tag}_a'], rtol=0, atol=1e-9)


CASES = dict(
    a=dict(nx=128, ny=128, patch=(64, 64), crop=8),
    b=dict(nx=128, ny=128, patch=(64, 64), crop=8, beam=True, umax=1.0, awin='hann'),
    c=dict(nx=64, ny=64, patch=(64, 64), crop=0),
    d=dict(nx=96, ny=128, patch=(48, 64), crop=4, beam=True, umax=1.0, T=16, levels=2),
    e=dict(nx=128, ny=128, patch=(64, 64), crop=8, gap=True),
    f=dict(nx=128, ny=128, patch=(64, 64), crop=8, pulses=True),
)


def _pulses(center):
    # 150 pulses about the track point abeam of the patch centre (the fixtures' 284 pulses are 0.55 m apart along y)
    mid = int(round(142 + float(center[1]) / 0.55))
    return max(0, mid - 75), min(284, mid + 75)


@pytest.mark.parametrize('tag', sorted(CASES))
def test_mosaic_matches_reference(g, tag):
    from fastsar_b200 import mosaic as mo
    kw = dict(CASES[tag])
    nx, ny = kw.pop('nx'), kw.pop('ny')
    if kw.pop('beam', False):
        kw['beam'] = _beam(g['ant'])
    if kw.pop('pulses', False):
        kw['pulses'] = _pulses
    fx, ant = _fx(g), g['ant']
    if kw.pop('gap', False):        # pulses dropped from the collection: the mosaic fills them with zero pulses
        keep = g['gap_keep']
        fx, ant = dict(fx, S=fx['S'][keep], ref=fx['ref'][keep]), ant[keep]
    info = []
    img = mo.form_mosaic(fx, ant, g['origin'], nx, ny, 0.5, 0.5, E1, E2, info=info, **kw)
    ref = g[f'img_{tag}']
    assert img.shape == ref.shape and img.dtype == np.complex64
    err = _rel_db(img, ref)
    print(f'mosaic {tag}: {err:.1f} dB against the reference')
    assert err < -75
    got = np.array([[i['pulses'][0], i['pulses'][1], i['K'], i['T'], i['sub'][0], i['sub'][1], i['levels'], i['df']]
                    for i in info])
    np.testing.assert_allclose(got, g[f'info_{tag}'], rtol=1e-12)


def test_mosaic_arguments(g):
    from fastsar_b200 import mosaic as mo
    fx = _fx(g)
    with pytest.raises(ValueError, match='exact'):
        mo.form_mosaic(fx, g['ant'], g['origin'], 64, 64, 0.5, 0.5, E1, E2, exact=True)
    with pytest.raises(ValueError, match='lacks'):
        mo.form_mosaic(dict(S=g['S']), g['ant'], g['origin'], 64, 64, 0.5, 0.5, E1, E2)
    with pytest.raises(ValueError, match='patch'):
        mo.form_mosaic(fx, g['ant'], g['origin'], 64, 64, 0.5, 0.5, E1, E2, patch=(0, 64))


def test_mosaic_without_shared_profiles(g, monkeypatch):
    """Where the shared range profiles would not fit the device, each patch takes the direct form: the same image
    as with them (the gate's edge samples aside), and the reference's within the same bar."""
    import torch
    from fastsar_b200 import mosaic as mo
    fx = _fx(g)
    with_prof = mo.form_mosaic(fx, g['ant'], g['origin'], 128, 128, 0.5, 0.5, E1, E2, patch=(64, 64), crop=8)
    monkeypatch.setattr(torch.cuda, 'mem_get_info', lambda *a, **k: (1 << 20, 1 << 30))
    direct = mo.form_mosaic(fx, g['ant'], g['origin'], 128, 128, 0.5, 0.5, E1, E2, patch=(64, 64), crop=8)
    print(f'mosaic without shared profiles: {_rel_db(direct, with_prof.astype(np.complex128)):.1f} dB from the shared '
          f'form, {_rel_db(direct, g["img_a"]):.1f} dB from the reference')
    assert _rel_db(direct, with_prof.astype(np.complex128)) < -70
    assert _rel_db(direct, g['img_a']) < -75
