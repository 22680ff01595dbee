"""The range gate on a B200 (ImageFormer(range_gate=...), fastsar/api.py:398-416 and 525-564): the gated history of
a seeded random history against the reference's (tests/golden/gate.npz), the gated image of a simulated wide-band
scene (an image 38 m across from a 24,000-sample collection: 195 samples kept) against the reference's gated image
and against the float64 exact backprojection of the whole history, 'auto' gating where the first level's filter
would not fit, and the errors the reference raises.
Tolerances: the gated history within 1e-5 of the reference's (float32 transforms of 30,000 samples); the image within
-70 dB of the reference former's (the parity bar), and against float64 64x of the whole history no further than the
reference former's gated image is (the factorized former's own error at this geometry, about -55 dB: its final
stage's predicted error is -57 dB)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden'))

GRID = dict(nx=96, ny=96, spx=0.4, spy=0.4, e1=(0.0, 1.0, 0.0), e2=(1.0, 0.0, 0.0))


def _rel_db(a, b):
    a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
    return float(10 * np.log10(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


@pytest.fixture(scope='module')
def wide():
    from make_golden import wide_band_collection, wide_band_scene
    from fastsar_b200 import sim
    col = wide_band_collection(sim)
    pos, amp = wide_band_scene()
    S = sim.simulate(col, pos, amp)
    return col, S


def test_gated_history_matches_reference(golden, wide):
    from fastsar_b200 import ImageFormer
    g = golden('gate')
    col, _ = wide
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, **GRID, range_gate=True)
    assert f.range_gate is not None and f.range_gate['kept'] == int(g['hist_kept'])
    rng = np.random.default_rng(21)
    S = (rng.standard_normal((col.Np, col.K)) + 1j * rng.standard_normal((col.Np, col.K))).astype(np.complex64)
    got = f._gate(torch.from_numpy(S).cuda())[:8].cpu().numpy()
    want = g['hist_gated']
    e = np.sqrt(np.sum(np.abs(got - want) ** 2) / np.sum(np.abs(want) ** 2))
    print(f'gated history: {f.range_gate["kept"]} of {col.K} samples, rel {e:.2e}')
    assert e < 1e-5


def test_gated_image_matches_reference_and_float64(golden, wide):
    from fastsar_b200 import ImageFormer, form_image
    from fastsar_b200.exact import backproject_device, plane_points
    g = golden('gate')
    col, S = wide
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, **GRID)                   # 'auto': the filter would not fit
    assert f.range_gate is not None and 'level kernel' in f.range_gate['note']
    assert f.levels == int(g['img_levels']) and f._plan['levels'][0]['Dk'] == int(g['img_Dk0'])
    img = f.form_device(S).cpu().numpy()
    e_ref = _rel_db(img, g['img'])
    pts = plane_points(GRID['nx'], GRID['ny'], GRID['spx'], GRID['spy'], GRID['e1'], GRID['e2'])
    ref64 = backproject_device(S, col.ant, col.fmin, col.df, pts, upsample=64).cpu().numpy()
    e64, e64_ref = _rel_db(img, ref64), _rel_db(g['img'], ref64)
    print(f'gated image ({f.range_gate["kept"]} of {col.K} samples): {e_ref:.1f} dB vs the reference former, '
          f'{e64:.1f} dB vs float64 64x of the whole history (the reference former\'s: {e64_ref:.1f} dB)')
    assert e_ref < -70.0
    assert e64 < -50.0 and e64 < e64_ref + 0.5
    assert np.array_equal(f(S.cpu().numpy()), img)
    assert np.array_equal(form_image(S.cpu().numpy(), col.ant, col.fmin, col.df, **GRID, range_gate=True), img)
    assert np.array_equal(f.form_many([S.cpu()])[0], img)


def test_range_gate_errors(wide):
    from fastsar_b200 import ImageFormer, sim
    col, S = wide
    with pytest.raises(ValueError, match='range_gate'):
        ImageFormer(col.ant, col.fmin, col.df, col.K, **GRID, range_gate='yes')
    with pytest.raises(ValueError, match='range_gate=True'):
        ImageFormer(col.ant, col.fmin, col.df, col.K, **GRID, range_gate=False)
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, **GRID, range_gate=True)
    bad = S.cpu().numpy().copy()
    bad[7, 100] = np.nan
    with pytest.raises(ValueError, match='non-finite.*pulse 7'):
        f(bad)
    with pytest.raises(ValueError, match='phase history must be'):
        f(S.cpu().numpy()[:, :-1])
    # an image that fills the swath is not gated
    small = sim.make_collect(res=0.5, scene=60.0, r0=5e3)
    assert ImageFormer(small.ant, small.fmin, small.df, small.K, 128, 128, 0.5, 0.5, range_gate=True).range_gate is None
