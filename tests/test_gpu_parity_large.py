"""Parity above the golden sizes, on a B200: the 4,096-pulse x 4,096-sample spotlight (the 512-pulse spotlight's
geometry, 9.6 GHz, 300 MHz, 600 km, 45 deg, 1.5 deg) formed to 2,048 x 2,048 pixels at 0.25 m, three levels of 16
and 4 children. The history is synthesized on the GPU (seeded targets, clutter at -30 dB, noise at -40 dB); the
reference's own CPU former (its ffbp_cpu.cpp kernels from oracle/_ref through the oracle's driver; the float64 port
where those are not built) forms the same image on the host cores.

* plain float32: within -70 dB of the reference former's image, no gain fitted, the peak within 1e-3 (the bar of
  fastsar tests/test_ffbp_cpu.py:34-38);
* the chosen form (precision='float16', learned taps, pmax 0.5): within -60 dB of the float64 exact backprojection at
  64x on 4,096 random pixels, no gain fitted."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


@pytest.fixture(scope='module')
def spot4k():
    from fastsar_b200 import sim
    w, S = sim.synthetic_history('spotlight_4k', seed=3, n_clutter=20000)
    return w, S


def test_spotlight4k_plain_matches_reference_former(spot4k, oracle_lib):
    from fastsar_b200 import ImageFormer
    w, S = spot4k
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2'])
    img = f.form_device(S).cpu().numpy()
    kind = 'reference' if oracle_lib.available('reference') else 'port'
    form, plan = oracle_lib.image_former(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'],
                                         w['e1'], w['e2'], kind=kind)
    assert plan['T'] == f.T and len(plan['levels']) == f.levels
    ref = form(S.cpu().numpy())
    e = oracle_lib.err_db(img, ref)
    peak = np.abs(img).max() / np.abs(ref).max()
    print(f'spotlight 4k, plain float32: {e:.1f} dB vs the reference former ({kind} kernels), peak ratio {peak:.6f}')
    assert e < -70.0 and abs(peak - 1) < 1e-3


def test_spotlight4k_chosen_form_against_float64(spot4k):
    from fastsar_b200 import ImageFormer
    from fastsar_b200.exact import backproject_device, plane_points
    w, S = spot4k
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2'],
                    precision='float16', taps='learned', pmax=0.5)
    img = f.form_device(S)
    idx = np.random.default_rng(9).choice(w['nx'] * w['ny'], 4096, replace=False)
    pts = plane_points(w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2']).reshape(-1, 3)[idx]
    ref = backproject_device(S, col.ant, col.fmin, col.df, pts, upsample=64).cpu().numpy()
    a = img.reshape(-1)[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.complex128)
    e = float(10 * np.log10(np.sum(np.abs(a - ref) ** 2) / np.sum(np.abs(ref) ** 2)))
    print(f'spotlight 4k, chosen form: {e:.1f} dB vs float64 exact backprojection 64x (no gain)')
    assert e < -60.0
