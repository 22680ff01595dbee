"""Parity of the CUDA path with the reference and the oracle, through the C ABI, on a B200.

* Stage kernels (ffbp_level, ffbp_final, ffbp_phases) against the oracle's float64 restatement of the reference's
  kernels on seeded inputs, including the edges the reference's tests exercise (levels that do not decimate along
  one axis, child counts that are not a multiple of a block's group, odd sizes, aperture weights).
* Whole images against the reference CPU former's images (tests/golden, no gain fitted; the bar of
  fastsar tests/test_ffbp_cpu.py:34-38: -70 dB and the peak within 1e-3) and against the oracle run here.
* The non-finite scan, bitwise repeatability, and the float64 phases against the planner's host float64 geometry.
Tolerances: the plain float32 path must be within -70 dB of the reference (the parity bar); kernels within 2e-5
relative of the float64 oracle."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


def _rel(a, b):
    a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def _dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.cuda() if dtype is None else t.to(dtype).cuda()


@pytest.fixture(scope='module')
def lib():
    from fastsar_b200 import _lib
    return _lib


def _level_case(rng, Np, P, K, C, Dk, Dp, pk=0.6, pp=0.5):
    from fastsar_b200 import plan as P_
    fk = P_.decimator_fir(K, Dk, pk)[0] if Dk > 1 else None
    fp = P_.decimator_fir(P, Dp, pp)[0] if Dp > 1 else None
    Ko = fk['n_out'] if fk else K
    Po = fp['n_out'] if fp else P
    x = (rng.standard_normal((Np, P, K)) + 1j * rng.standard_normal((Np, P, K))).astype(np.complex64)
    c0 = rng.uniform(-0.5, 0.5, (Np, C, P)).astype(np.float32)
    sl = rng.uniform(-0.01, 0.01, (Np, C, P)).astype(np.float32)
    return x, c0, sl, fk, fp, Ko, Po


def _run_level_gpu(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, window=None, bad=None):
    L = lib.load()
    Np, P, K = x.shape
    C = c0.shape[1]
    ph = np.stack([c0, sl], axis=-1).astype(np.float32)
    dx, dph = _dev(x), _dev(ph)
    tk = _dev(np.asarray(fk['kern'], np.float32)) if fk else None
    tp = _dev(np.asarray(fp['kern'], np.float32)) if fp else None
    wp = _dev(window[0]) if window is not None else None
    wk = _dev(window[1]) if window is not None else None
    out = torch.zeros((Np * C, Po, Ko), dtype=torch.complex64, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    lib.check(L.ffbp_level(dx.data_ptr(), Np, P, K, dph.data_ptr(), C, lib.tptr(tk), fk['L'] if fk else 1,
                           fk['pl'] if fk else 0, Dk, Ko, (K - 1) / 2.0, lib.tptr(tp), fp['L'] if fp else 1,
                           fp['pl'] if fp else 0, Dp, Po, lib.tptr(wp), lib.tptr(wk), out.data_ptr(),
                           lib.tptr(bad), s), 'ffbp_level')
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, window=None):
    L = oracle_lib.lib('port')
    Np, P, K = x.shape
    C = c0.shape[1]
    if window is not None:
        x = (x * (window[0][:, None] * window[1][None, :]).astype(np.float32)[None]).astype(np.complex64)
    taps = np.asarray(fk['kern'], np.float32) if fk else np.ones(1, np.float32)
    yre = np.zeros((Np * C, P, Ko), np.float32)
    yim = np.zeros_like(yre)
    L.rot_fir_k_cplx(np.ascontiguousarray(x).view(np.float32), Np, P, K, c0, sl, C, taps, fk['L'] if fk else 1,
                     fk['pl'] if fk else 0, Dk, Ko, (K - 1) / 2.0, yre, yim)
    if fp is None:
        return yre + 1j * yim
    zre = np.zeros((Np * C, Po, Ko), np.float32)
    zim = np.zeros_like(zre)
    L.fir_p(yre, yim, Np * C, P, Ko, np.asarray(fp['kern'], np.float32), fp['L'], fp['pl'], Dp, Po, zre, zim)
    return zre + 1j * zim


LEVEL_CASES = [
    # Np, P, K, C, Dk, Dp
    (1, 300, 520, 8, 3, 4),      # a first level: one parent, both axes decimated
    (3, 97, 131, 5, 2, 3),       # C not a multiple of the block's 4 children, odd sizes
    (2, 64, 90, 4, 1, 2),        # no frequency decimation (Dk = 1)
    (2, 80, 200, 6, 4, 1),       # no pulse decimation (Dp = 1)
    (1, 50, 700, 2, 7, 2),       # a long frequency FIR (Lk > 100)
    (4, 40, 60, 3, 1, 1),        # rotation only
]


@pytest.mark.parametrize('case', LEVEL_CASES, ids=[f'Np{c[0]}-P{c[1]}-K{c[2]}-C{c[3]}-Dk{c[4]}-Dp{c[5]}' for c in LEVEL_CASES])
def test_level_kernel_matches_oracle(lib, oracle_lib, case):
    Np, P, K, C, Dk, Dp = case
    rng = np.random.default_rng(sum(case))
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, Np, P, K, C, Dk, Dp)
    got = _run_level_gpu(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    e = _rel(got, ref)
    print(f'level {case}: rel {e:.2e}')
    assert e < 2e-5, e


def test_level_kernel_window_and_nonfinite(lib, oracle_lib):
    rng = np.random.default_rng(3)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 120, 256, 4, 3, 2)
    from fastsar_b200.api import _window
    w = _window(120, 256)
    got = _run_level_gpu(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    assert _rel(got, ref) < 2e-5
    x[0, 77, 5] = np.nan
    x[0, 90, 100] = np.inf
    bad = torch.full((1,), 2 ** 31 - 1, dtype=torch.int32, device='cuda')
    _run_level_gpu(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w, bad=bad)
    assert int(bad.item()) == 77


def _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, window=None, bad=None, opts=None):
    """ffbp_level_tc (ffbp_level_tc_ex with launch options opts: a dict of ffbp_tc_opts fields) on the device;
    -> (output, status [err, amax_in, amax_out] as ints)."""
    L = lib.load()
    Np, P, K = x.shape
    C = c0.shape[1]
    ph = np.stack([c0, sl], axis=-1).astype(np.float32)
    dx, dph = _dev(x), _dev(ph)
    tk = _dev(np.asarray(fk['kern'], np.float32)) if fk else None
    tp = _dev(np.asarray(fp['kern'], np.float32)) if fp else None
    wp = _dev(window[0]) if window is not None else None
    wk = _dev(window[1]) if window is not None else None
    out = torch.zeros((Np * C, Po, Ko), dtype=torch.complex64, device='cuda')
    nbytes = int(L.ffbp_level_tc_scratch_bytes(Np, C, P, Ko))
    scratch = torch.empty(nbytes // 4 + 4, dtype=torch.int32, device='cuda')
    status = torch.zeros(3, dtype=torch.int32, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    args = (dx.data_ptr(), Np, P, K, dph.data_ptr(), C, lib.tptr(tk), fk['L'] if fk else 1, fk['pl'] if fk else 0, Dk,
            Ko, (K - 1) / 2.0, lib.tptr(tp), fp['L'] if fp else 1, fp['pl'] if fp else 0, Dp, Po, lib.tptr(wp),
            lib.tptr(wk), out.data_ptr(), lib.tptr(bad), scratch.data_ptr(), nbytes, status.data_ptr())
    if opts is None:
        lib.check(L.ffbp_level_tc(*args, s), 'ffbp_level_tc')
    else:
        o = lib.TcOpts(*(int(opts.get(k, 0)) for k in ('nt', 'sb', 'copies', 'repeat', 'fir', 'consumers')))
        lib.check(L.ffbp_level_tc_ex(*args, ctypes.byref(o), s), 'ffbp_level_tc_ex')
    torch.cuda.synchronize()
    return out.cpu().numpy(), status.cpu().numpy()


TC_LEVEL_CASES = [
    # Np, P, K, C, Dk, Dp, frequency pass fraction
    (1, 300, 520, 8, 3, 4, 0.6),      # a first level, few children (most accumulator rows idle)
    (3, 97, 131, 5, 2, 3, 0.6),       # odd sizes, several parents
    (2, 64, 90, 4, 1, 2, 0.6),        # no frequency decimation (Dk = 1: one tap)
    (2, 80, 200, 6, 4, 1, 0.6),       # no pulse decimation (Dp = 1)
    (1, 200, 900, 64, 3, 10, 0.6),    # 64 children (every accumulator row), several column tiles
    (2, 120, 700, 56, 7, 8, 0.45),    # 56 children, 57 frequency taps
    (8, 90, 160, 30, 5, 6, 0.6),      # many parents, 30 children
    (3, 70, 700, 12, 9, 4, 0.45),     # 12 children, 73 taps (accumulator rows repeated: lane quarters 1, 3 idle)
    (2, 60, 500, 32, 6, 5, 0.45),     # 32 children, the most with the rows repeated
    (2, 100, 800, 56, 9, 8, 0.45),    # 73 frequency taps (K padded to 80)
    (1, 90, 1200, 40, 10, 6, 0.5),    # 90 frequency taps (K padded to 96)
]


@pytest.mark.parametrize('fir', [0, 2], ids=['fir-default', 'fir-tensor-cores'])
@pytest.mark.parametrize('case', TC_LEVEL_CASES,
                         ids=[f'Np{c[0]}-P{c[1]}-K{c[2]}-C{c[3]}-Dk{c[4]}-Dp{c[5]}' for c in TC_LEVEL_CASES])
def test_level_tensor_cores_match_oracle(lib, oracle_lib, case, fir):
    """The tensor-core level against the float64 oracle of the reference's rot_fir_k + fir_p: the products in split
    bfloat16 (about 2^-16) and the float16 intermediate (11 significant bits) leave a relative error near 2^-12;
    the bar is 1e-3 (-60 dB). The output's largest component is recorded exactly. The pulse FIR on its default
    kernel (the CUDA cores at these sizes) and on the tensor cores (a banded product with float16 hi + lo taps)."""
    Np, P, K, C, Dk, Dp, pk = case
    rng = np.random.default_rng(sum(case[:6]) + 11)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, Np, P, K, C, Dk, Dp, pk=pk)
    got, st = _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, opts=dict(fir=fir) if fir else None)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    e = _rel(got, ref)
    print(f'tensor-core level {case} fir {fir}: rel {e:.2e} ({20 * np.log10(e):.1f} dB)')
    assert st[0] == 0
    assert e < 1e-3, e
    amax_out = np.frombuffer(np.int32(st[2]).tobytes(), np.float32)[0]
    assert amax_out == np.max(np.abs(got.view(np.float32)))
    amax_in = np.frombuffer(np.int32(st[1]).tobytes(), np.float32)[0]
    assert amax_in == np.max(np.abs(x.view(np.float32)))


TC_OPTS_CASES = [TC_LEVEL_CASES[i] for i in (0, 4, 6, 7, 10)]


@pytest.mark.parametrize('case', TC_OPTS_CASES,
                         ids=[f'Np{c[0]}-P{c[1]}-K{c[2]}-C{c[3]}-Dk{c[4]}-Dp{c[5]}' for c in TC_OPTS_CASES])
def test_level_tensor_cores_launch_options_same_bits(lib, case):
    """The launch options (ffbp_tc_opts: columns per tile, B stages, plane copies, row repeat, the pulse FIR's
    kernel) change the schedule, not the arithmetic: plane copies and B stages give the default's output bit for bit;
    columns per tile and the row repeat move the points where the consumers seed the output ramp's recurrence (about
    1e-7), which can flip a rounding of the float16 intermediate (one unit: 5e-4 of that value), and the two pulse
    FIR kernels sum in different orders (the tensor cores with the taps as float16 hi + lo): within 1e-4 of the
    default; a set that does not fit is refused with FFBP_E_UNSUPPORTED (ValueError)."""
    Np, P, K, C, Dk, Dp, pk = case
    rng = np.random.default_rng(sum(case[:6]) + 11)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, Np, P, K, C, Dk, Dp, pk=pk)
    want, _ = _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp)
    AP = -(-(fp['L'] if fp else 1) // Dp)
    default_fir = 2 if (Po >= 512 or AP > 12) else 1            # the launcher's default for the pulse FIR's kernel
    sets = [dict(copies=4), dict(copies=2), dict(nt=32), dict(nt=64, copies=4), dict(nt=96), dict(nt=128, sb=2),
            dict(sb=3), dict(repeat=1, nt=16), dict(repeat=1, nt=48, copies=4), dict(repeat=1, nt=80), dict(nt=48),
            dict(fir=1), dict(fir=2), dict(fir=1, copies=4), dict(consumers=4), dict(consumers=4, nt=48, copies=4),
            dict(consumers=4, repeat=1, nt=80), dict(consumers=8), dict(consumers=12), dict(consumers=12, nt=48),
            dict(consumers=12, nt=96, copies=4)]
    ran = 0
    for o in sets:
        try:
            got, st = _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, Dk, Dp, opts=o)
        except ValueError as e:
            assert 'columns per tile' in str(e) or 'B stages' in str(e), (o, str(e))
            continue
        assert st[0] == 0
        if set(o) <= {'copies', 'sb'} or o == dict(fir=default_fir) or o == dict(consumers=8):
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), o
        else:
            assert _rel(got, want) < 1e-4, (o, _rel(got, want))
        ran += 1
    print(f'{case}: {ran} of {len(sets)} option sets ran')
    assert ran >= 5


def test_level_tensor_cores_long_pulse_filter(lib, oracle_lib):
    """A pulse filter spanning more than 12 output pulses (Dp 2, pass fraction 0.9: 45 outputs per input pulse), which
    only the tensor-core pulse FIR takes (the launcher's default there), against the float64 oracle; the CUDA-core
    kernel refuses it with FFBP_E_UNSUPPORTED."""
    rng = np.random.default_rng(21)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 2, 120, 300, 8, 3, 2, pp=0.9)
    assert -(-fp['L'] // 2) > 12
    got, st = _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, 3, 2)
    e = _rel(got, ref)
    print(f'long pulse filter (Lp {fp["L"]}): rel {e:.2e}')
    assert st[0] == 0 and e < 1e-3
    with pytest.raises(ValueError, match='12 output pulses'):
        _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, opts=dict(fir=1))


def test_level_tensor_cores_window_nonfinite_and_limits(lib, oracle_lib):
    """The first level's window and the non-finite scan on the tensor-core level, and the shapes it leaves to the
    float32 kernel (more than 96 frequency taps) refused with FFBP_E_UNSUPPORTED."""
    rng = np.random.default_rng(5)
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 120, 256, 12, 3, 2)
    from fastsar_b200.api import _window
    w = _window(120, 256)
    got, st = _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    ref = _oracle_level_full(oracle_lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w)
    assert _rel(got, ref) < 1e-3
    x[0, 77, 5] = np.nan
    x[0, 90, 100] = np.inf
    bad = torch.full((1,), 2 ** 31 - 1, dtype=torch.int32, device='cuda')
    _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, 3, 2, window=w, bad=bad)
    assert int(bad.item()) == 77
    x, c0, sl, fk, fp, Ko, Po = _level_case(rng, 1, 50, 1200, 2, 11, 2)     # Lk = 121
    with pytest.raises(ValueError, match='96'):
        _run_level_tc(lib, x, c0, sl, fk, fp, Ko, Po, 11, 2)


@pytest.mark.parametrize('T', [16, 32])
@pytest.mark.parametrize('weighted', [False, True])
def test_final_kernel_matches_oracle(lib, oracle_lib, T, weighted):
    rng = np.random.default_rng(T + weighted)
    B, Pf, Qf = 5, 13, 57
    d = (rng.standard_normal((B, Pf, Qf)) + 1j * rng.standard_normal((B, Pf, Qf))).astype(np.complex64)
    ux, uy = rng.uniform(-0.9, 0.9, (B, Pf)), rng.uniform(-0.9, 0.9, (B, Pf))
    spx, spy = 0.3, 0.45
    a0, a1, fc2 = 64.1, 0.013, 64.4
    ucx, ucy, rc = rng.uniform(-0.5, 0.5, B), rng.uniform(-0.5, 0.5, B), rng.uniform(4e3, 6e3, B)
    w = np.stack([rng.uniform(0.5, 1.5, (B, Pf)), rng.uniform(-0.01, 0.01, (B, Pf)),
                  rng.uniform(-0.01, 0.01, (B, Pf))]).astype(np.float32) if weighted else None
    L = lib.load()
    out = torch.zeros((B, T, T), dtype=torch.complex64, device='cuda')
    dd = [_dev(a) for a in (d, ux, uy, ucx, ucy, rc)]
    dw = _dev(w) if weighted else None
    lib.check(L.ffbp_final(dd[0].data_ptr(), B, Pf, Qf, T, dd[1].data_ptr(), dd[2].data_ptr(), spx, spy, a0, a1,
                           dd[3].data_ptr(), dd[4].data_ptr(), dd[5].data_ptr(), fc2, lib.tptr(dw), 0, out.data_ptr(),
                           torch.cuda.current_stream().cuda_stream), 'ffbp_final')
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    O = oracle_lib.lib('port')
    dlx = (np.arange(T) - (T - 1) / 2.0) * spx
    dly = (np.arange(T) - (T - 1) / 2.0) * spy
    ore = np.zeros((B, T, T), np.float32)
    oim = np.zeros_like(ore)
    wp = [None] * 3 if w is None else [np.ascontiguousarray(x) for x in w]
    O.final_tiles(np.ascontiguousarray(d.real), np.ascontiguousarray(d.imag), B, Pf, Qf, T, ux, uy, dlx, dly, a0, a1,
                  ucx, ucy, rc, fc2, ore, oim, *[None if x is None else x.ctypes.data for x in wp])
    e = _rel(got, ore + 1j * oim)
    print(f'final T={T} weighted={weighted}: rel {e:.2e}')
    assert e < 2e-5, e


def test_phases_match_host_float64(lib, golden):
    """The device float64 phases of the first two levels against the planner's host float64 (collection_arrays)."""
    from fastsar_b200 import plan as P_
    from fastsar_b200.sim import Collect
    rec = golden('plan_spot512')
    fmin, df, K, nx, ny, spx, spy, T, nlev, pmax = rec['scal']
    col = Collect(fmin=fmin, df=df, K=int(K), ant=rec['ant'], res=0.5)
    plan = P_.make_plan(col, int(nx), int(ny), spx, spy, T=int(T), nlev=int(nlev), pmax=pmax, e1=rec['e1'], e2=rec['e2'])
    coll = P_.collection_arrays(plan, col.ant)
    L = lib.load()
    for i in range(2):
        lv = plan['levels'][i]
        B = lv['ref'].shape[0]
        out = torch.zeros((B, lv['C'], lv['P'], 2), dtype=torch.float32, device='cuda')
        ant, ref, cen = _dev(lv['ant']), _dev(lv['ref']), _dev(lv['cen'])
        kc = (lv['K'] - 1) / 2.0
        k0c, k1 = 2.0 * (lv['f0'] + kc * lv['df']) / 299792458.0, 2.0 * lv['df'] / 299792458.0
        lib.check(L.ffbp_phases(ant.data_ptr(), lv['P'], ref.data_ptr(), B, cen.data_ptr(), lv['C'], None, k0c, k1, 0,
                                out.data_ptr(), torch.cuda.current_stream().cuda_stream), 'ffbp_phases')
        torch.cuda.synchronize()
        g = out.cpu().numpy()
        dc0 = np.abs(g[..., 0] - coll['levels'][i]['c0'])
        dc0 = np.minimum(dc0, 1 - dc0)                   # a wrap at +-0.5 cycles
        assert dc0.max() < 1e-6
        np.testing.assert_allclose(g[..., 1], coll['levels'][i]['slope'], rtol=1e-6, atol=1e-9)


# ------------------------------------------------------------------------------------------------ whole images

def _former(golden, nlev, **kw):
    from fastsar_b200 import ImageFormer
    g = golden('image_small')
    fmin, df, K = g['scal']
    return ImageFormer(g['ant'], fmin, df, int(K), 128, 128, 0.5, 0.5, T=16, levels=nlev, **kw), g


@pytest.mark.parametrize('nlev', [2, 3])
def test_image_matches_reference_former(golden, oracle_lib, nlev):
    """The reference's CPU test scene (fastsar tests/test_ffbp_cpu.py:10-38): -70 dB and the peak within 1e-3 of the
    reference former's image, no gain fitted."""
    f, g = _former(golden, nlev)
    img = f(g['S'])
    ref = g[f'ffbp_l{nlev}']
    e = oracle_lib.err_db(img, ref)
    peak = np.abs(img).max() / np.abs(ref).max()
    print(f'{nlev} levels: {e:.1f} dB vs reference former, peak ratio {peak:.6f}')
    assert e < -70.0 and abs(peak - 1) < 1e-3


def test_image_without_window(golden, oracle_lib):
    f, g = _former(golden, 3, window=False)
    assert oracle_lib.err_db(f(g['S']), g['ffbp_l3_nowin']) < -70.0


def test_spotlight512_matches_reference_and_fp64(golden, oracle_lib):
    """The 512-pulse, 600 km spotlight (32 targets, clutter -30 dB, noise -40 dB): against the reference former's
    image, and against the reference's float64 64x backprojection on 4,096 pixels."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'])
    assert f.T == int(g['T'])
    img = f(g['S'])
    e = oracle_lib.err_db(img, g['ffbp'])
    e64 = oracle_lib.rel_db(img.ravel()[g['bp64_idx']], g['bp64'])
    print(f'spotlight 512: {e:.1f} dB vs reference former; {e64:.1f} dB vs float64 BP 64x')
    assert e < -70.0
    assert e64 < -55.0


def test_repeatable_bitwise(golden):
    f, g = _former(golden, 3)
    a = f(g['S'])
    b = f(g['S'])
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_nonfinite_history_raises(golden):
    f, g = _former(golden, 2)
    S = g['S'].copy()
    S[123, 7] = np.nan
    with pytest.raises(ValueError, match='pulse 123'):
        f(S)


def test_torch_input_matches_numpy(golden):
    f, g = _former(golden, 2)
    a = f(g['S'])
    b = f.form_device(torch.from_numpy(g['S']).cuda()).cpu().numpy()
    assert np.array_equal(a, b)


# ------------------------------------------------------------------------------------------------ tensor-core final

@pytest.mark.parametrize('mode,tol,T', [(2, 2e-4, 32), (1, 3e-3, 32), (1, 3e-3, 16)], ids=['bf16x3', 'f16', 'f16-t16'])
@pytest.mark.parametrize('weighted', [False, True])
@pytest.mark.parametrize('shape', [(5, 13, 57), (300, 7, 96), (3, 40, 130), (4, 1, 40), (301, 38, 71), (400, 59, 113)],
                         ids=['small', 'many-tiles', 'long-q', 'one-subaperture', 'spotlight-12k-final', 'two-stages'])
def test_final_tensor_cores_match_oracle(lib, oracle_lib, mode, tol, T, weighted, shape):
    """The tcgen05 final stage against the float64 oracle: split bfloat16 products within 2e-4, one float16 product
    within 3e-3 (its operands carry 11 bits), T = 32 and (float16) T = 16; units beyond one per multiprocessor, tile
    counts that leave a float16 unit part-filled (two T = 32 or four T = 16 tiles a unit), one final subaperture (one
    MMA issuer), padding of Qf to a multiple of 16, aperture weights, the chosen form's final stage shape at the
    12,288 x 8,832 spotlight (Pf 38, Qf 71), and a shape whose operands leave room for two pipeline stages only, with
    an odd subaperture count and several units per block."""
    rng = np.random.default_rng(7 * mode + weighted + shape[0])
    B, Pf, Qf = shape
    d = (rng.standard_normal((B, Pf, Qf)) + 1j * rng.standard_normal((B, Pf, Qf))).astype(np.complex64)
    ux, uy = rng.uniform(-0.9, 0.9, (B, Pf)), rng.uniform(-0.9, 0.9, (B, Pf))
    spx, spy = 0.3, 0.45
    a0, a1, fc2 = 64.1, 0.013, 64.4
    ucx, ucy, rc = rng.uniform(-0.5, 0.5, B), rng.uniform(-0.5, 0.5, B), rng.uniform(4e3, 6e3, B)
    w = np.stack([rng.uniform(0.5, 1.5, (B, Pf)), rng.uniform(-0.01, 0.01, (B, Pf)),
                  rng.uniform(-0.01, 0.01, (B, Pf))]).astype(np.float32) if weighted else None
    L = lib.load()
    out = torch.zeros((B, T, T), dtype=torch.complex64, device='cuda')
    dd = [_dev(a) for a in (d, ux, uy, ucx, ucy, rc)]
    dw = _dev(w) if weighted else None
    lib.check(L.ffbp_final(dd[0].data_ptr(), B, Pf, Qf, T, dd[1].data_ptr(), dd[2].data_ptr(), spx, spy, a0, a1,
                           dd[3].data_ptr(), dd[4].data_ptr(), dd[5].data_ptr(), fc2, lib.tptr(dw), mode,
                           out.data_ptr(), torch.cuda.current_stream().cuda_stream), 'ffbp_final')
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    O = oracle_lib.lib('port')
    dlx = (np.arange(T) - (T - 1) / 2.0) * spx
    dly = (np.arange(T) - (T - 1) / 2.0) * spy
    ore = np.zeros((B, T, T), np.float32)
    oim = np.zeros_like(ore)
    wp = [None] * 3 if w is None else [np.ascontiguousarray(x) for x in w]
    O.final_tiles(np.ascontiguousarray(d.real), np.ascontiguousarray(d.imag), B, Pf, Qf, T, ux, uy, dlx, dly, a0, a1,
                  ucx, ucy, rc, fc2, ore, oim, *[None if x is None else x.ctypes.data for x in wp])
    e = _rel(got, ore + 1j * oim)
    print(f'tensor-core final mode {mode} {shape} weighted={weighted}: rel {e:.2e}')
    assert e < tol, e


def test_image_tensor_cores_match_reference(golden, oracle_lib, monkeypatch):
    """The 512-pulse spotlight (T = 32) with the split-bfloat16 tensor-core final stage against the reference former's
    image: within the -70 dB parity bar."""
    from fastsar_b200 import ImageFormer, sim
    monkeypatch.setenv('FASTSAR_FINAL', 'tc3')
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'])
    img = f(g['S'])
    e = oracle_lib.err_db(img, g['ffbp'])
    e64 = oracle_lib.rel_db(img.ravel()[g['bp64_idx']], g['bp64'])
    print(f'float32/tc3: {e:.1f} dB vs reference former; {e64:.1f} dB vs float64 BP 64x')
    assert e < -70.0


@pytest.mark.parametrize('T', ['auto', 16])
def test_image_mixed_precision_against_float64(golden, oracle_lib, T):
    """precision='float16' (tensor-core levels and final stage, 80 dB filters) on the 512-pulse spotlight, with the
    chosen tile size (32 here) and with T = 16 (four tiles per tensor-core unit): its error against the float64 exact
    backprojection (64x) is below -60 dB and no worse than the reference former's own (its 70 dB filters put it
    -66.8 dB from the float64 image); against the reference former's image the two formers' filter errors add."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision='float16', T=T)
    assert f.T == (32 if T == 'auto' else T)
    img = f(g['S'])
    e = oracle_lib.err_db(img, g['ffbp'])
    e64 = oracle_lib.rel_db(img.ravel()[g['bp64_idx']], g['bp64'])
    eref = oracle_lib.rel_db(g['ffbp'].ravel()[g['bp64_idx']], g['bp64'])
    print(f'float16 T={f.T}: {e64:.1f} dB vs float64 BP 64x (reference former {eref:.1f} dB); {e:.1f} dB vs reference former')
    assert e64 < -60.0
    assert e64 < eref + 0.5
    assert e < -50.0


@pytest.mark.parametrize('precision,final', [('float32', 'tc3'), ('float16', 'fp32')], ids=['bf16x3', 'f16'])
def test_image_tensor_cores_repeatable_bitwise(golden, monkeypatch, precision, final):
    """Two MMA issuers accumulate fixed subsets of the final subapertures into their own accumulators, summed in a
    fixed order: the tensor-core image is the same bits on every call."""
    from fastsar_b200 import ImageFormer, sim
    monkeypatch.setenv('FASTSAR_FINAL', final)
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision=precision)
    a = f(g['S'])
    b = f(g['S'])
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_image_tuned_levels_match_default(golden):
    """ImageFormer(tune_levels=True) times the tensor-core levels' launch options per level shape when it is built
    and plans with the fastest: every tuned level records its choice, and the image is the default's to within 3e-4
    relative (-70 dB; the chosen form itself is about -64 dB from float64): the options move the seeding of the
    output ramp's recurrence, and with it a float16 rounding here and there, and the pulse FIR's kernel (on the tensor
    cores its operands are split into float16 halves) rounds differently from the CUDA-core one (1.0e-4 measured with
    the tensor-core FIR on all three levels)."""
    from fastsar_b200 import ImageFormer, sim, tune
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    args = (col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'])
    f = ImageFormer(*args, precision='float16', tune_levels=True)
    assert f.level_opts is not None and len(f.level_opts) == f.levels
    assert all(o is not None for o in f.level_opts)
    print('tuned level options:', f.level_opts)
    a = f(g['S'])
    b = ImageFormer(*args, precision='float16')(g['S'])
    print(f'tuned against default: {_rel(a, b):.1e}')
    assert _rel(a, b) < 3e-4, _rel(a, b)
    # a second former of the same shapes takes the options from the cache
    n = len(tune._LEVEL_CACHE)
    ImageFormer(*args, precision='float16', tune_levels=True).release()
    assert len(tune._LEVEL_CACHE) == n


def test_image_float16_large_amplitudes(golden, oracle_lib):
    """The float16 operands and intermediates are scaled by powers of two from the data's largest component: a
    history 2^24 times larger (corner reflectors and the coherent gain of a large image reach far beyond float16's
    65504) gives a finite image equal to 2^24 times the image of the original history, whose error against the
    float64 exact backprojection stays below -60 dB."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision='float16')
    big = float(2 ** 24)
    img = f((g['S'] * big).astype(np.complex64))
    assert np.all(np.isfinite(img.view(np.float32)))
    small = f(g['S'])
    r = _rel(img / big, small)
    e64 = oracle_lib.rel_db(img.ravel()[g['bp64_idx']] / big, g['bp64'])
    print(f'float16 at 2^24 x amplitude: {r:.1e} from the unscaled image; {e64:.1f} dB vs float64 BP 64x')
    assert r < 1e-6
    assert e64 < -60.0


def test_form_many_matches_device_forming(golden):
    """ImageFormer.form_many (ffbp_form_host: uploads and downloads on their own streams, two images in flight) gives
    bit for bit the images of form_device, for page-locked and pageable host histories, float32 and the tensor-core
    form; a history with a non-finite sample raises naming that history and its pulse."""
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    rng = np.random.default_rng(3)
    Ss = [g['S'].astype(np.complex64)] + [(g['S'] * (rng.standard_normal() + 1j * rng.standard_normal())).astype(np.complex64)
                                          for _ in range(4)]
    for prec in ('float32', 'float16'):
        f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision=prec)
        want = [f.form_device(torch.from_numpy(S).cuda()).cpu().numpy() for S in Ss]
        pinned = [torch.from_numpy(S).pin_memory() for S in Ss]
        got = f.form_many(pinned)
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
        got = f.form_many(Ss[:3])                               # pageable numpy histories
        assert all(np.array_equal(a, b) for a, b in zip(got, want[:3]))
        bad = [S.copy() for S in Ss[:3]]
        bad[2][37, 5] = np.nan
        with pytest.raises(ValueError, match='phase history 2 .*pulse 37'):
            f.form_many(bad)
