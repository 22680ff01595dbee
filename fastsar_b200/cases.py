"""A profiling harness, not part of the former's API: single-stage cases of a workload's plan, for timing one kernel
at a time and for small profiler captures (the commands of profiles/*.md run it):

    python -m fastsar_b200.cases level L1 [--parents 8] [--pulses 2048] [--form tc|fused|fp32] [--fir 0|1|2] [--taps learned|80|70]
    python -m fastsar_b200.cases final [--tiles 20000] [--mode f16|bf16x3|fp32] [--taps learned|80|70]
    python -m fastsar_b200.cases exact [--workload spotlight_4k] [--interp cubic|linear] [--pulses 1024]
    python -m fastsar_b200.cases products [--side 4096] [--window 7]

`level`: one merge stage of the plan (its children, decimations and filters) on `--parents` parents of random
samples and random child phases, through ffbp_level_tc (tensor cores in two passes: level_tc_gemm and level_fir),
ffbp_level_fused (tensor cores in one pass) or ffbp_level (float32: level_kernel); `--pulses` shortens the pulse
axis (the pulse filter is then
designed for the shorter axis by the same rule). `final`: the final stage through ffbp_final on `--tiles` tiles of
the plan's final shape with random samples and geometry. Each prints the event-timed duration of every repetition.
The defaults are the 16,384 x 8,192 -> 12,288 x 8,832 spotlight (workload spotlight_12k) planned as the chosen form
(learned taps, pmax 0.5); --pmax 0.4 --taps 70 gives the reference's plan.
"""
import argparse
import ctypes

import numpy as np

from . import _lib
from . import plan as _plan
from . import sim


def workload_plan(name='spotlight_12k', taps='learned', pmax=0.5):
    """The plan of a named workload with learned taps ('learned', Kaiser-sinc fallback at 80 dB) or Kaiser-sinc
    filters at the given attenuation, at oversampling parameter pmax (0.5: the chosen form's; 0.4: the
    reference's default)."""
    w = sim.workload(name)
    model = None
    atten = 80.0
    if taps == 'learned':
        from .learned import LearnedTaps
        model = LearnedTaps.load()
    else:
        atten = float(taps)
    return w, _plan.make_plan(w['col'], w['nx'], w['ny'], w['spx'], w['spy'], T=32, nlev=3, pmax=pmax, atten=atten,
                              e1=w['e1'], e2=w['e2'], taps=model)


def level_case(level, parents, pulses=0, form='tc', taps='learned', reps=3, seed=1, pmax=0.5, fir=0, opts=None):
    import torch
    L = _lib.load()
    w, pl = workload_plan(taps=taps, pmax=pmax)
    lv = pl['levels'][level]
    P, K, C, Ko, Po, Dk, Dp = lv['P'], lv['K'], lv['C'], lv['Ko'], lv['Po'], lv['Dk'], lv['Dp']
    fk, fp = lv['fir_k'], lv['fir_p']
    if pulses:
        P = int(pulses)
        if lv['kind_p'] == 'learned':
            from .learned import LearnedTaps
            fp = LearnedTaps.load().decimator(P, Dp, min(lv['pass_p'], 0.95), level, 1)[0]
        else:
            fp = _plan.decimator_fir(P, Dp, min(lv['pass_p'], 0.95), lv['dec_p'][3])[0]
        Po = fp['n_out']
    g = torch.Generator(device='cuda')
    g.manual_seed(seed)
    x = torch.view_as_complex(torch.randn((parents, P, K, 2), device='cuda', generator=g)).contiguous()
    ph = torch.stack([torch.rand((parents, C, P), device='cuda', generator=g) - 0.5,
                      (torch.rand((parents, C, P), device='cuda', generator=g) - 0.5) * 0.004], -1).contiguous()
    tk = torch.tensor(np.asarray(fk['kern'], np.float32), device='cuda')
    tp = torch.tensor(np.asarray(fp['kern'], np.float32), device='cuda')
    out = torch.empty((parents * C, Po, Ko), dtype=torch.complex64, device='cuda')
    st = torch.zeros(3, dtype=torch.int32, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    nb = int(L.ffbp_level_tc_scratch_bytes(parents, C, P, Ko))
    scr = torch.empty(nb // 4 + 4, dtype=torch.int32, device='cuda') if form == 'tc' else None

    def run():
        if form == 'fused':
            _lib.check(L.ffbp_level_fused(x.data_ptr(), parents, P, K, ph.data_ptr(), C, tk.data_ptr(), fk['L'],
                                          fk['pl'], Dk, Ko, (K - 1) / 2.0, tp.data_ptr(), fp['L'], fp['pl'], Dp, Po,
                                          None, None, out.data_ptr(), None, st.data_ptr(), s), 'ffbp_level_fused')
        elif form == 'tc':
            oo = dict(opts or {}, **({'fir': int(fir)} if fir else {}))
            o = _lib.TcOpts(*(int(oo.get(k, 0)) for k in ('nt', 'sb', 'copies', 'repeat', 'fir', 'consumers')))
            _lib.check(L.ffbp_level_tc_ex(x.data_ptr(), parents, P, K, ph.data_ptr(), C, tk.data_ptr(), fk['L'],
                                          fk['pl'], Dk, Ko, (K - 1) / 2.0, tp.data_ptr(), fp['L'], fp['pl'], Dp, Po, None,
                                          None, out.data_ptr(), None, scr.data_ptr(), nb, st.data_ptr(),
                                          ctypes.byref(o), s), 'ffbp_level_tc_ex')
        else:
            _lib.check(L.ffbp_level(x.data_ptr(), parents, P, K, ph.data_ptr(), C, tk.data_ptr(), fk['L'], fk['pl'], Dk,
                                    Ko, (K - 1) / 2.0, tp.data_ptr(), fp['L'], fp['pl'], Dp, Po, None, None,
                                    out.data_ptr(), None, s), 'ffbp_level')
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        print(f'level {level} ({form}, taps {taps}) parents={parents} P={P} K={K} C={C} Ko={Ko} Po={Po} '
              f'Lk={fk["L"]} Lp={fp["L"]}: {e0.elapsed_time(e1):.3f} ms', flush=True)


def final_case(tiles, mode='f16', taps='learned', reps=2, seed=2, pmax=0.5):
    import torch
    L = _lib.load()
    w, pl = workload_plan(taps=taps, pmax=pmax)
    f = pl['final']
    Pf, Qf, T = f['P'], f['K'], pl['T']
    m = {'fp32': _lib.FFBP_FINAL_FP32, 'f16': _lib.FFBP_FINAL_TC_F16, 'bf16x3': _lib.FFBP_FINAL_TC_BF16X3}[mode]
    g = torch.Generator(device='cuda')
    g.manual_seed(seed)
    d = torch.view_as_complex(torch.randn((tiles, Pf, Qf, 2), device='cuda', generator=g)).contiguous()
    ux = (torch.rand((tiles, Pf), device='cuda', generator=g, dtype=torch.float64) - 0.5) * 0.1
    uy = (torch.rand((tiles, Pf), device='cuda', generator=g, dtype=torch.float64) - 0.5) * 1.6
    ucx, ucy = ux.mean(1).contiguous(), uy.mean(1).contiguous()
    rc = torch.full((tiles,), 5e5, device='cuda', dtype=torch.float64)
    out = torch.empty((tiles, T, T), dtype=torch.complex64, device='cuda')
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(L.ffbp_final(d.data_ptr(), tiles, Pf, Qf, T, ux.data_ptr(), uy.data_ptr(), 0.2, 0.2, 64.0, 0.0085,
                                ucx.data_ptr(), ucy.data_ptr(), rc.data_ptr(), 64.5, None, m, out.data_ptr(), s),
                   'ffbp_final')
        e1.record()
        torch.cuda.synchronize()
        print(f'final ({mode}, taps {taps}) tiles={tiles} Pf={Pf} Qf={Qf} T={T}: {e0.elapsed_time(e1):.3f} ms',
              flush=True)


def exact_case(workload='spotlight_4k', interp='cubic', pulses=1024, reps=5):
    """ExactFormer's tiled backprojection alone (ffbp_exact_backproject) on one chunk of a workload's pulses: the
    seeded synthetic history padded, windowed and inverse-transformed once, then the kernel timed."""
    import ctypes
    import torch
    from .exact import ExactFormer
    L = _lib.load()
    w, S = sim.synthetic_history(workload, seed=1, n_clutter=20000)
    col = w['col']
    f = ExactFormer(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2'],
                    interp=interp, chunk=pulses)
    d = f._upload()
    n = min(f.chunk, f.P)
    st = torch.cuda.current_stream().cuda_stream
    pad = torch.zeros((n, f.nfft), dtype=torch.complex64, device='cuda')
    _lib.check(L.ffbp_exact_pad(S[:n].data_ptr(), n, f.K, d['wp'].data_ptr(), d['wk'].data_ptr(), f.nfft,
                                pad.data_ptr(), None, 0, st), 'ffbp_exact_pad')
    prof = torch.fft.ifft(pad, dim=1).contiguous()
    e1, e2 = (ctypes.c_double * 3)(*f.e1), (ctypes.c_double * 3)(*f.e2)
    out = torch.zeros((f.nx, f.ny), dtype=torch.complex64, device='cuda')
    for r in range(reps + 1):
        e0, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check(L.ffbp_exact_backproject(prof.data_ptr(), n, f.nfft, d['ant'].data_ptr(), d['ref'].data_ptr(),
                                            d['cen'].data_ptr(), f.ntx, f.nty, f.tx, f.ty, f.nx, f.ny, f.spx, f.spy,
                                            e1, e2, f.inv_dr, f.kcyc, int(f.cubic), f.along1, None, out.data_ptr(),
                                            st), 'ffbp_exact_backproject')
        e1_.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1_)
        if r:
            print(f'exact {workload} {interp} tile {f.tile}, {n} pulses: {ms:.3f} ms, '
                  f'{f.nx * f.ny * n / (ms * 1e-3) / 1e9:.0f} GBP/s', flush=True)


def products_case(side=4096, window=7, reps=3, seed=3):
    """The stack products' pixel kernels alone on two seeded complex images side x side on the device: the coherence
    map (window x window), the detected image's box mean in dB (box 5), a running-average step and the 32 x 32 tile
    statistics, each event-timed with the bytes it must move (GB/s)."""
    import torch
    L = _lib.load()
    g = torch.Generator(device='cuda').manual_seed(seed)
    a = torch.randn((side, side), dtype=torch.complex64, device='cuda', generator=g)
    b = torch.randn((side, side), dtype=torch.complex64, device='cuda', generator=g)
    out = torch.empty((side, side), dtype=torch.float32, device='cuda')
    acc, wacc = torch.empty_like(out), torch.empty_like(out)
    tm, tv = torch.empty(max((side // 32) ** 2, 1), device='cuda'), torch.empty(max((side // 32) ** 2, 1), device='cuda')
    st = torch.cuda.current_stream().cuda_stream
    n = side * side
    cases = [
        ('coherence_kernel', 20 * n, lambda: L.ffbp_coherence(a.data_ptr(), b.data_ptr(), side, side, window, window,
                                                              out.data_ptr(), st)),
        ('box_kernel', 12 * n, lambda: L.ffbp_box_mean(a.data_ptr(), _lib.PIX_POWER, side, side, 5, 1, out.data_ptr(), st)),
        ('mean_add_kernel', 24 * n, lambda: L.ffbp_mean_add(a.data_ptr(), _lib.PIX_POWER, n, 1.0, 1.0, 0, acc.data_ptr(),
                                                            wacc.data_ptr(), st)),
        ('tile_stats_kernel', 4 * n, lambda: L.ffbp_tile_stats(out.data_ptr(), side, side, 32, 1.0, tm.data_ptr(),
                                                               tv.data_ptr(), st)),
    ]
    for name, nbytes, fn in cases:
        for r in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(fn(), name)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if r:
                print(f'{name} {side} x {side}: {ms:.3f} ms, {nbytes / (ms * 1e-3) / 1e9:.0f} GB/s', flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description='time one stage of a workload plan')
    ap.add_argument('stage', choices=('level', 'final', 'exact', 'products'))
    ap.add_argument('level', nargs='?', default='L1', choices=('L0', 'L1', 'L2'))
    ap.add_argument('--parents', type=int, default=8)
    ap.add_argument('--pulses', type=int, default=0)
    ap.add_argument('--form', choices=('tc', 'fused', 'fp32'), default='tc')
    ap.add_argument('--fir', type=int, choices=(0, 1, 2), default=0,
                    help="tc: the pulse FIR's kernel (0 the launcher's default, 1 CUDA cores, 2 tensor cores)")
    ap.add_argument('--opts', default=None,
                    help='tc: launch options as JSON, e.g. \'{"consumers": 4, "copies": 4, "nt": 80}\'')
    ap.add_argument('--tiles', type=int, default=20000)
    ap.add_argument('--mode', choices=('f16', 'bf16x3', 'fp32'), default='f16')
    ap.add_argument('--taps', default='learned', help="'learned' or a Kaiser-sinc attenuation in dB (70, 80)")
    ap.add_argument('--reps', type=int, default=3)
    ap.add_argument('--pmax', type=float, default=0.5)
    ap.add_argument('--workload', default='spotlight_4k', help='exact: the workload')
    ap.add_argument('--interp', choices=('cubic', 'linear'), default='cubic', help='exact: the interpolation')
    ap.add_argument('--side', type=int, default=4096, help='products: the images\' side')
    ap.add_argument('--window', type=int, default=7, help='products: the coherence window')
    a = ap.parse_args(argv)
    if a.stage == 'products':
        products_case(a.side, a.window, a.reps)
    elif a.stage == 'exact':
        exact_case(a.workload, a.interp, a.pulses or 1024, a.reps)
    elif a.stage == 'level':
        import json
        level_case(int(a.level[1]), a.parents, a.pulses, a.form, a.taps, a.reps, pmax=a.pmax, fir=a.fir,
                   opts=json.loads(a.opts) if a.opts else None)
    else:
        final_case(a.tiles, a.mode, a.taps, a.reps, pmax=a.pmax)


if __name__ == '__main__':
    main()
