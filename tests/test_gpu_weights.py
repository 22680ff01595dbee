"""ImageFormer(aperture_weight=...) on a B200 against the reference's CPU former with the same weight
(tests/golden/weights.npz, written by tests/golden/make_golden.py from fastsar/api.py:203-244 and the C++ former):
a pixel- and pulse-dependent weight applied per final subaperture with its gradients (fastsar/ffbp_cpu.cpp:302-469
takes w0, gx, gyr); within the -70 dB parity bar with no gain fitted."""
import numpy as np
import pytest

from test_plan import weight_fn

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


@pytest.mark.parametrize('nlev', [2, 3])
def test_aperture_weight_matches_reference_former(golden, oracle_lib, nlev):
    from fastsar_b200 import ImageFormer
    g, img = golden('weights'), golden('image_small')
    fmin, df, K = img['scal']
    P = img['ant'].shape[0]
    f = ImageFormer(img['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=nlev, window=False,
                    aperture_weight=weight_fn(P))
    got = f(img['S'])
    ref = g[f'img_l{nlev}']
    e = oracle_lib.err_db(got, ref)
    peak = np.abs(got).max() / np.abs(ref).max()
    print(f'aperture weight, {nlev} levels: {e:.1f} dB vs the reference former, peak ratio {peak:.6f}')
    assert e < -70.0 and abs(peak - 1) < 1e-3
    # and the weight matters: the unweighted image is far from the weighted one
    plain = ImageFormer(img['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=nlev, window=False)(img['S'])
    assert oracle_lib.err_db(plain, ref) > -30.0
