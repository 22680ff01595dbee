"""BatchFormer on a B200: patches of uneven sizes from two collections (the 512-pulse spotlight and the reference's
small CPU test case), float32 and the tensor-core form (T = 32 and 16), captured into one CUDA graph (ffbp_batch_create) and formed
by one launch, give bit for bit the images each former forms alone; a non-finite sample is reported with its
history's index; a range-gated former is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


def _patches(golden):
    """(former, history) pairs: patches at offsets c of the spotlight (antenna positions - c, each pulse referenced
    to its range to the scene origin) and of the small case."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    r0 = np.linalg.norm(col.ant, axis=1)
    out = []
    for (cx, cy), (nx, ny), prec in [((0.0, 0.0), (64, 96), 'float32'), ((20.0, -15.0), (128, 128), 'float16'),
                                     ((-30.0, 10.0), (96, 200), 'float32'), ((5.0, 25.0), (256, 64), 'float32'),
                                     ((-10.0, -20.0), (160, 160), 'float16')]:
        c = np.array([cy, cx, 0.0])
        f = ImageFormer(col.ant - c, col.fmin, col.df, col.K, nx, ny, 0.25, 0.25, w['e1'], w['e2'], ref=r0,
                        precision=prec)
        out.append((f, g['S']))
    s = golden('image_small')
    fmin, df, K = s['scal']
    out.append((ImageFormer(s['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=3), s['S']))
    out.append((ImageFormer(s['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=3, precision='float16'), s['S']))
    return out


def test_batch_matches_formers_alone(golden):
    from fastsar_b200 import BatchFormer
    pairs = _patches(golden)
    want = [f.form_device(torch.from_numpy(np.ascontiguousarray(S, np.complex64)).cuda()).cpu().numpy() for f, S in pairs]
    batch = BatchFormer([f for f, _ in pairs])
    got = batch([S for _, S in pairs])
    for i, (a, b) in enumerate(zip(got, want)):
        assert a.shape == b.shape and np.array_equal(a, b), i
    # a second launch on the same buffers gives the same images
    again = [m.cpu().numpy() for m in batch.form_device()]
    assert all(np.array_equal(a, b) for a, b in zip(again, want))
    hs = [np.ascontiguousarray(S, np.complex64).copy() for _, S in pairs]
    hs[3][11, 7] = np.nan
    with pytest.raises(ValueError, match='phase history 3 .*pulse 11'):
        batch(hs)
    # the spotlight's patches sharing one device history
    shared = BatchFormer([f for f, _ in pairs], sources=[0, 0, 0, 0, 0, 1, 1])
    got = shared([pairs[0][1], pairs[-1][1]])
    assert all(np.array_equal(a, b) for a, b in zip(got, want))
    with pytest.raises(ValueError, match='differ'):
        BatchFormer([f for f, _ in pairs], sources=[0, 0, 0, 0, 0, 0, 0])


def test_batch_refuses_gated_formers():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden'))
    from make_golden import wide_band_collection
    from fastsar_b200 import BatchFormer, ImageFormer, sim
    col = wide_band_collection(sim)
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 96, 96, 0.4, 0.4, (0.0, 1.0, 0.0), (1.0, 0.0, 0.0))
    assert f.range_gate is not None
    with pytest.raises(ValueError, match='gates its history'):
        BatchFormer([f])
