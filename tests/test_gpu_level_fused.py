"""The one-pass tensor-core level (ffbp_level_fused: the products on the tensor cores, the ramp and the pulse FIR's
running sums in tensor memory) against the float64 oracle of the reference's rot_fir_k + fir_p, through the C ABI,
on a B200; and whole images formed with it against the two-pass form and the float64 exact backprojection.

Tolerances: the products are split bfloat16 (hi hi + hi lo + lo hi: about 2^-16 per product) accumulated in float32,
and nothing is rounded to float16 on the way, so the level is within 1e-4 relative of the float64 oracle."""
import numpy as np
import pytest

from test_gpu_parity import _dev, _level_case, _oracle_level_full, _rel

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


@pytest.fixture(scope='module')
def lib():
    from fastsar_b200 import _lib
    return _lib


def _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, window=None, bad=None):
    """ffbp_level_fused on the device -> (output, status [err, unused, amax_out] as ints)."""
    L = lib.load()
    Np, P, K = x.shape
    C = c0.shape[1]
    ph = np.stack([c0, sl], axis=-1).astype(np.float32)
    dx, dph = _dev(x), _dev(ph)
    tk = _dev(np.asarray(fk['kern'], np.float32)) if fk else None
    tp = _dev(np.asarray(fp['kern'], np.float32)) if fp else None
    wp = _dev(window[0]) if window is not None else None
    wk = _dev(window[1]) if window is not None else None
    out = torch.full((Np * C, Po, Ko), complex(np.nan, np.nan), dtype=torch.complex64, device='cuda')
    status = torch.zeros(3, dtype=torch.int32, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    lib.check(L.ffbp_level_fused(dx.data_ptr(), Np, P, K, dph.data_ptr(), C, lib.tptr(tk), fk['L'] if fk else 1,
                                 fk['pl'] if fk else 0, Dk, Ko, (K - 1) / 2.0, lib.tptr(tp), fp['L'] if fp else 1,
                                 fp['pl'] if fp else 0, Dp, Po, lib.tptr(wp), lib.tptr(wk), out.data_ptr(),
                                 lib.tptr(bad), status.data_ptr(), s), 'ffbp_level_fused')
    torch.cuda.synchronize()
    return out.cpu().numpy(), status.cpu().numpy()


FUSED_CASES = [
    # Np, P, K, C, Dk, Dp, frequency pass fraction
    (1, 300, 520, 8, 3, 4, 0.6),      # a first level, few children
    (3, 97, 131, 5, 2, 3, 0.6),       # odd sizes, several parents
    (2, 64, 90, 4, 1, 2, 0.6),        # no frequency decimation (Dk = 1: one tap)
    (2, 80, 200, 6, 4, 1, 0.6),       # no pulse decimation (Dp = 1: one running sum)
    (1, 600, 900, 64, 3, 10, 0.6),    # 64 children, 32-column tiles, several output segments
    (2, 120, 700, 56, 7, 8, 0.45),    # 56 children, 57 frequency taps
    (8, 90, 160, 30, 5, 6, 0.6),      # many parents, 30 children: 64-column tiles, rows repeated
    (3, 70, 700, 12, 9, 4, 0.45),     # 12 children, 73 taps
    (2, 60, 500, 32, 6, 5, 0.45),     # 32 children, the most with the rows repeated
    (2, 100, 800, 33, 9, 8, 0.45),    # 33 children (32-column tiles, quarter 2 partly idle), 73 taps
    (1, 90, 1200, 40, 10, 6, 0.5),    # 90 frequency taps (K padded to 96)
    (1, 2000, 300, 16, 2, 12, 0.6),   # a long pulse axis: many output segments with their halos
]


@pytest.mark.parametrize('case', FUSED_CASES,
                         ids=[f'Np{c[0]}-P{c[1]}-K{c[2]}-C{c[3]}-Dk{c[4]}-Dp{c[5]}' for c in FUSED_CASES])
def test_level_fused_matches_oracle(lib, oracle_lib, case):
    Np, P, K, C, Dk, Dp, pk = case
    rng = np.random.default_rng(sum(case[:6]) + 23)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, Np, P, K, C, Dk, Dp, pk=pk, pp=0.35)
    assert fp is None or -(-fp['L'] // Dp) <= 8        # the pulse FIR feeds at most 8 outputs per input
    got, st = _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    assert np.all(np.isfinite(got.view(np.float32))), 'outputs left unwritten'
    e = _rel(got, ref)
    print(f'one-pass level {case}: rel {e:.2e} ({20 * np.log10(e):.1f} dB)')
    assert st[0] == 0
    assert e < 1e-4, e
    amax_out = np.frombuffer(np.int32(st[2]).tobytes(), np.float32)[0]
    assert amax_out == np.max(np.abs(got.view(np.float32)))


def test_level_fused_window_nonfinite_and_limits(lib, oracle_lib):
    """The first level's window and the non-finite scan, and the shapes the one-pass kernel refuses (more than 96
    frequency taps; a pulse FIR spanning more than 8 output pulses) with FFBP_E_UNSUPPORTED."""
    rng = np.random.default_rng(5)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 120, 256, 12, 3, 2, pp=0.35)
    from fastsar_b200.api import _window
    w = _window(120, 256)
    got, _ = _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    assert _rel(got, ref) < 1e-4
    x[0, 77, 5] = np.nan
    x[0, 90, 100] = np.inf
    bad = torch.full((1,), 2 ** 31 - 1, dtype=torch.int32, device='cuda')
    _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w, bad=bad)
    assert int(bad.item()) == 77
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 50, 1200, 2, 11, 2, pp=0.35)     # Lk = 121
    with pytest.raises(ValueError, match='96'):
        _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, 11, 2)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 400, 64, 2, 1, 4, pp=0.95)   # a pulse FIR of 87 outputs
    assert -(-fp['L'] // 4) > 8
    with pytest.raises(ValueError, match='8 outputs'):
        _run_level_fused(lib, x, c0, sl, fk, fp, Ko, Po, 1, 4)


def _spot512(precision, monkeypatch, levels):
    from fastsar_b200 import ImageFormer, sim
    monkeypatch.setenv('FASTSAR_LEVELS', levels)
    w = sim.workload('spotlight_512')
    col = w['col']
    return ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision=precision,
                       taps='learned', pmax=0.5)


def test_image_one_pass_levels(golden, oracle_lib, monkeypatch):
    """The 512-pulse spotlight formed with the one-pass levels: within -60 dB of the float64 exact backprojection
    (no gain fitted), no worse than the two-pass form (whose float16 intermediate it does without), and the same
    bits on every call."""
    g = golden('image_spot512')
    f1 = _spot512('float16', monkeypatch, 'tc1')
    assert any(k == 'level_tc' for k, _, _ in f1._dev.form_profile(torch.from_numpy(g['S']).cuda(),
                                                                    torch.empty((512, 512), dtype=torch.complex64,
                                                                                device='cuda')))
    a = f1(g['S'])
    b = f1(g['S'])
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    f2 = _spot512('float16', monkeypatch, 'tc2')
    c = f2(g['S'])
    e1 = oracle_lib.err_db(a.ravel()[g['bp64_idx']], g['bp64'])
    e2 = oracle_lib.err_db(c.ravel()[g['bp64_idx']], g['bp64'])
    d = oracle_lib.err_db(a, c)
    print(f'one-pass levels: {e1:.1f} dB vs float64 BP 64x; two-pass {e2:.1f} dB; one-pass vs two-pass {d:.1f} dB')
    assert e1 < -60.0
    assert e1 < e2 + 0.5
