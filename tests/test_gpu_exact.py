"""The device oracle family against the CPU oracle: the float64 point backprojection (ffbp_bp_points_f64) against
oracle.backproject_fp64, monostatic and bistatic, and the float64 phase-history synthesis (ffbp_simulate) against the
host float64 direct sum."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


def test_simulate_matches_host_float64():
    from fastsar_b200 import sim
    rng = np.random.default_rng(5)
    col = sim.make_collect(res=0.5, scene=40.0, r0=20e3)
    pos = np.stack([rng.uniform(-15, 15, 300), rng.uniform(-15, 15, 300), rng.uniform(-2, 2, 300)], 1)
    amp = rng.standard_normal(300) + 1j * rng.standard_normal(300)
    got = sim.simulate(col, pos, amp, chunk=128).cpu().numpy()        # several launches accumulate
    ref = sim.simulate_brute(col, pos, amp)
    e = np.sqrt(np.sum(np.abs(got - ref) ** 2) / np.sum(np.abs(ref) ** 2))
    print(f'simulate: rel {e:.2e}')
    assert e < 2e-6


@pytest.mark.parametrize('bistatic', [False, True])
def test_fp64_backprojection_matches_oracle(golden, oracle_lib, bistatic):
    from fastsar_b200.exact import backproject_device, plane_points
    g = golden('image_small')
    fmin, df, K = g['scal']
    ant = g['ant']
    rcv = ant + np.array([0.0, 0.0, 100.0]) if bistatic else None
    pts = plane_points(64, 48, 0.5, 0.5, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0))
    got = backproject_device(g['S'], ant, fmin, df, pts, rcv=rcv, upsample=64).cpu().numpy()
    ref = oracle_lib.backproject_fp64(g['S'], ant, fmin, df, pts, rcv=rcv, upsample=64)
    e = oracle_lib.err_db(got, ref)
    print(f'fp64 BP (bistatic={bistatic}): {e:.1f} dB against the oracle')
    assert e < -120.0


# ------------------------------------------------------------------------------------------------- ExactFormer
@pytest.mark.parametrize('interp,bar', [('cubic', -80.0), ('linear', -80.0)])
def test_exact_former_matches_reference(golden, oracle_lib, interp, bar):
    """ExactFormer (tiled exact backprojection on the GPU) against the reference's ExactFormer(backend='cpu') on the
    128 x 128 test scene (tests/golden/image_small.npz): the same algorithm in float32 with the same tiles, windows
    and interpolation, so the images agree far below either one's error against the float64 backprojection (no gain
    fitted); and that error itself, cubic at upsample 8 below -60 dB."""
    from fastsar_b200 import ExactFormer
    g = golden('image_small')
    fmin, df, K = g['scal']
    f = ExactFormer(g['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, interp=interp)
    img = f(g['S'])
    ref = g[f'exact_{interp}']
    e = 20 * np.log10(np.linalg.norm(img - ref) / np.linalg.norm(ref))
    e64 = oracle_lib.err_db(img, g['bp64'])
    print(f'ExactFormer {interp}: {e:.1f} dB vs the reference ExactFormer, {e64:.1f} dB vs float64 BP 64x, tile {f.tile}')
    assert e < bar
    if interp == 'cubic':
        assert e64 < -60.0


def test_exact_former_torch_input_nonfinite_and_form_image(golden):
    from fastsar_b200 import ExactFormer, form_image
    g = golden('image_small')
    fmin, df, K = g['scal']
    f = ExactFormer(g['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5)
    a = f(g['S'])
    b = f(torch.from_numpy(g['S']).cuda())
    assert np.array_equal(a, b)
    c = form_image(g['S'], g['ant'], fmin, df, 128, 128, 0.5, 0.5, algorithm='bp')
    assert np.array_equal(a, c)
    S = g['S'].copy()
    S[37, 5] = np.inf
    with pytest.raises(ValueError, match='pulse 37'):
        f(S)


def test_exact_former_close_range_tiles(golden):
    """A grid at 1 km picks 16 x 16 tiles: the image against the float64 backprojection of its pixels."""
    from fastsar_b200 import ExactFormer, sim
    from fastsar_b200.exact import backproject, plane_points
    col = sim.make_collect(res=0.5, scene=60.0, r0=1e3)
    rng = np.random.default_rng(11)
    pos = np.stack([rng.uniform(-20, 20, 12), rng.uniform(-15, 15, 12), np.zeros(12)], 1)
    amp = rng.standard_normal(12) + 1j * rng.standard_normal(12)
    S = sim.simulate_brute(col, pos, amp).astype(np.complex64)
    f = ExactFormer(col.ant, col.fmin, col.df, col.K, 96, 80, 0.5, 0.5)
    assert f.tile == (16, 16)
    img = f(S)
    ref = backproject(S, col.ant, col.fmin, col.df, plane_points(96, 80, 0.5, 0.5), upsample=64)
    g_ = np.vdot(img, ref) / np.vdot(img, img)
    e = 20 * np.log10(np.linalg.norm(g_ * img - ref) / np.linalg.norm(ref))
    print(f'ExactFormer at 1 km, 16 x 16 tiles: {e:.1f} dB vs float64 BP 64x')
    assert e < -55.0
