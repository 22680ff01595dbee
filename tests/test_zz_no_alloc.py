"""ffbp_form_static, the form call for callers that cannot allocate device memory when they form an image (a device
memory pool they do not control, a real-time loop that must stay out of the CUDA allocator): its scratch is a static
device array of the library, so the call allocates nothing. Checked through the C ABI against ffbp_form on a
caller-allocated workspace, bit for bit, on two calls in a row (the array keeps the previous call's contents), for
the float32 and the tensor-core forms, and for its refusal of a plan whose workspace exceeds the array. This module
is collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


def _form_static(dev, S, img):
    from fastsar_b200 import _lib
    L = _lib.load()
    bad = ctypes.c_int(-2)
    rc = L.ffbp_form_static(dev.handle, ctypes.c_void_p(S.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(bad))
    _lib.check(rc, 'ffbp_form_static')
    return bad.value


@pytest.mark.parametrize('nlev', [2, 3])
def test_static_workspace_matches_allocated_workspace(golden, nlev):
    from fastsar_b200 import ImageFormer
    g = golden('image_small')
    fmin, df, K = g['scal']
    f = ImageFormer(g['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=nlev)
    assert f._dev.ws_bytes <= 64 << 20
    S = torch.from_numpy(g['S']).cuda()
    ref = f.form_device(S).cpu().numpy()
    for _ in range(2):
        img = torch.full((128, 128), complex(np.nan, np.nan), dtype=torch.complex64, device='cuda')
        assert _form_static(f._dev, S, img) == -1
        # the same kernels on the same inputs: the same bits
        assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    # a history with a non-finite sample is reported through the static path too
    Sb = S.clone()
    Sb[17, 3] = complex(np.inf, 0.0)
    img = torch.empty((128, 128), dtype=torch.complex64, device='cuda')
    assert _form_static(f._dev, Sb, img) == 17


def test_static_workspace_tensor_core_form(golden):
    """The mixed-precision form (tensor-core levels, whose float16 intermediate lives in the workspace, and the
    tensor-core final stage) of the 512-pulse spotlight: its workspace fits the static array, and the static call
    gives the same bits as ffbp_form on an allocated workspace, twice in a row."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision='float16')
    assert f._dev.ws_bytes <= 64 << 20
    S = torch.from_numpy(g['S']).cuda()
    ref = f.form_device(S).cpu().numpy()
    for _ in range(2):
        img = torch.full((512, 512), complex(np.nan, np.nan), dtype=torch.complex64, device='cuda')
        assert _form_static(f._dev, S, img) == -1
        assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_static_workspace_refuses_a_large_plan():
    from fastsar_b200 import ImageFormer, sim
    w = sim.workload('spotlight_4k')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2'])
    assert f._dev.ws_bytes > 64 << 20
    S = torch.zeros((col.Np, col.K), dtype=torch.complex64, device='cuda')
    img = torch.empty((w['nx'], w['ny']), dtype=torch.complex64, device='cuda')
    with pytest.raises(ValueError, match='static workspace'):
        _form_static(f._dev, S, img)
