"""The autotuner of a patch's plan: build a former for each candidate (levels, tile size, precision, taps, pmax),
drop those that cannot be built or formed or whose predicted final-stage error misses the target, time the rest on the patch's history
with CUDA events and keep the fastest. No counterpart in the reference, which plans every patch by fixed rules
(fastsar/patches.py:162-171 for the levels, fastsar/ffbp2.py:300-307 for the tile size).

    former, choice, table = tune_former(make, candidates, S_dev, target_db=-60.0)

make(**kwargs) -> ImageFormer; candidates: a list of kwargs; S_dev: the patch's history on the device.
"""
import json
import os

import numpy as np

from . import plan as _plan

CHOSEN = [dict(precision='float16', taps='learned', pmax=0.5, T=t, levels=lv) for t in (16, 32) for lv in (2, 3, 4)]
FLOAT32 = [dict(precision='float32', taps='learned', T=t, levels=lv) for t in (16, 32) for lv in (2, 3, 4)]


def predicted_error_db(f, T):
    """The final stage's predicted error (dB) of a former's geometry at tile size T (fastsar/ffbp2.py:276-297)."""
    lv0 = f._plan['levels'][0]
    fmax = float(lv0['f0']) + lv0['K'] * float(lv0['df'])
    return float(_plan.final_phase_error(f.ant, fmax, f.nx, f.ny, f._plan['spx'], f._plan['spy'], f._plan['e1'],
                                         f._plan['e2'], T))


def time_former(f, S_dev, reps=3):
    """Median device time (ms) of reps formations after one warm-up."""
    import torch
    out = torch.empty((f.nx, f.ny), dtype=torch.complex64, device=S_dev.device)
    f.form_device(S_dev, out, check=False)
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        f.form_device(S_dev, out, check=False)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    f.check()                                        # a candidate whose pipeline aborted is not timed as a success
    return float(np.median(ts))


def tune_former(make, candidates, S_dev, target_db=-60.0, reps=3):
    """The fastest former among the candidates whose predicted final-stage error meets target_db (the one with the
    smallest predicted error when none does) -> (former, kwargs, table [(kwargs, predicted dB, ms or reason)])."""
    import torch
    table, best, fallback = [], None, None
    for kw in candidates:
        try:
            f = make(**kw)
        except (ValueError, RuntimeError) as e:
            table.append((kw, None, f'not built: {str(e)[:60]}'))
            continue
        err = predicted_error_db(f, f.T)
        if err > target_db:
            table.append((kw, err, 'misses the target'))
            if fallback is None or err < fallback[1]:
                fallback = (kw, err)
            f.release()
            del f
            continue
        try:
            ms = time_former(f, S_dev, reps)
        except (ValueError, RuntimeError, MemoryError) as e:   # a shape a kernel refuses, an abort, no memory
            table.append((kw, err, f'not formed: {str(e)[:60]}'))
            f.release()
            del f
            continue
        table.append((kw, err, ms))
        if best is None or ms < best[2]:
            if best is not None:
                best[0].release()
            best = (f, kw, ms)
        else:
            f.release()
        del f
        torch.cuda.empty_cache()
    if best is None:
        if fallback is None:
            raise ValueError('no candidate plan could be built for this patch')
        return make(**fallback[0]), fallback[0], table
    return best[0], best[1], table


# ------------------------------------------------------------------------------------------- level launch options

# Tuned launch options by level signature. Seeded from the packaged file (fastsar_b200/data/level_opts.json, made by
# `python -m fastsar_b200.tune --workload ...` on a B200) or from FASTSAR_TUNE_CACHE when set, which also receives
# every new result; in-process otherwise.
_LEVEL_CACHE = {}
_CACHE_LOADED = False
PACKAGED_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data', 'level_opts.json')


def _cache_path():
    return os.environ.get('FASTSAR_TUNE_CACHE') or None


def _key(sig):
    return ','.join(str(v) for v in sig)


def _load_cache():
    global _CACHE_LOADED
    if _CACHE_LOADED:
        return
    _CACHE_LOADED = True
    for path in (PACKAGED_CACHE, _cache_path()):
        if path and os.path.exists(path):
            with open(path) as f:
                for k, v in json.load(f).get('levels', {}).items():
                    _LEVEL_CACHE[tuple(int(x) for x in k.split(','))] = v


def _save_cache(path):
    doc = dict(device='B200 (sm_100a)', note='tensor-core level launch options by level signature: parents, children, '
               'frequency decimation, frequency taps, input samples, input pulses, output samples, output pulses, '
               'pulse decimation, pulse taps (fastsar_b200.tune.level_signature)',
               levels={_key(k): v for k, v in sorted(_LEVEL_CACHE.items()) if v is not None})
    tmp = path + '.tmp'
    with open(tmp, 'w') as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def level_signature(lv, Np):
    """What a tensor-core level's timing depends on: its shapes and filter lengths."""
    Lk = lv['fir_k']['L'] if lv['fir_k'] is not None else 1
    Lp = lv['fir_p']['L'] if lv['fir_p'] is not None else 1
    return (int(Np), int(lv['C']), int(lv['Dk']), int(Lk), int(lv['K']), int(lv['P']), int(lv['Ko']), int(lv['Po']),
            int(lv['Dp']), int(Lp))


def _level_candidates(C, Lk):
    """Launch option sets of a tensor-core level in the order a coordinate search visits them: the pulse FIR's kernel
    (CUDA or tensor cores), plane copies, consumer warps (8, 4 or 12; 16 less them copy Hankel rows), then columns per
    tile (the multiples of 8 x consumer warps / 4 that the launcher takes), then the row repeat off, then the B
    stages."""
    Lkp = ((max(Lk, 1) + 15) // 16) * 16
    rep_ok = Lkp > 32 and C <= 32
    return dict(fir=[1, 2], copies=[2, 4], consumers=[8, 4, 12],
                nt={8: list(range(32, 129, 32)), 4: list(range(16, 129, 16)), 12: list(range(24, 129, 24))},
                nt16=list(range(16, 129, 16)), repeat_off=rep_ok, sb=[2, 3, 4])


def tune_level(lv, Np, reps=3, max_parents=1024, seed=0):
    """The fastest launch options (ffbp_tc_opts as a dict) of one tensor-core level's first pass, timed with CUDA
    events on random samples and child phases of the level's shapes and its own filters (at most max_parents
    parents: the timing is linear in them beyond a few waves), by a coordinate search from the defaults. Results are
    cached by level_signature. -> (opts, table [(opts, ms or reason)]); opts None when the level is not a
    tensor-core level."""
    import ctypes
    import torch
    from . import _lib
    _load_cache()
    key = level_signature(lv, Np)
    if key in _LEVEL_CACHE:
        return _LEVEL_CACHE[key], []
    L = _lib.load()
    n = int(min(Np, max_parents))
    C, P, K, Ko, Po, Dk, Dp = (int(lv[k]) for k in ('C', 'P', 'K', 'Ko', 'Po', 'Dk', 'Dp'))
    fk, fp = lv['fir_k'], lv['fir_p']
    Lk = fk['L'] if fk is not None else 1
    g = torch.Generator(device='cuda')
    g.manual_seed(seed)
    x = torch.view_as_complex(torch.randn((n, P, K, 2), device='cuda', generator=g)).contiguous()
    ph = torch.stack([torch.rand((n, C, P), device='cuda', generator=g) - 0.5,
                      (torch.rand((n, C, P), device='cuda', generator=g) - 0.5) * 0.004], -1).contiguous()
    tk = torch.tensor(np.asarray(fk['kern'], np.float32), device='cuda') if fk is not None else None
    tp = torch.tensor(np.asarray(fp['kern'], np.float32), device='cuda') if fp is not None else None
    out = torch.empty((n * C, Po, Ko), dtype=torch.complex64, device='cuda')
    st = torch.zeros(3, dtype=torch.int32, device='cuda')
    nb = int(L.ffbp_level_tc_scratch_bytes(n, C, P, Ko))
    scr = torch.empty(nb // 4 + 4, dtype=torch.int32, device='cuda')
    stream = torch.cuda.current_stream().cuda_stream
    ptr = lambda t: None if t is None else t.data_ptr()

    def run(o):
        opts = _lib.TcOpts(*(int(o.get(k, 0)) for k in ('nt', 'sb', 'copies', 'repeat', 'fir', 'consumers')))
        _lib.check(L.ffbp_level_tc_ex(x.data_ptr(), n, P, K, ph.data_ptr(), C, ptr(tk), Lk,
                                      fk['pl'] if fk is not None else 0, Dk, Ko, (K - 1) / 2.0, ptr(tp),
                                      fp['L'] if fp is not None else 1, fp['pl'] if fp is not None else 0, Dp, Po,
                                      None, None, out.data_ptr(), None, scr.data_ptr(), nb, st.data_ptr(),
                                      ctypes.byref(opts), stream), 'ffbp_level_tc_ex')

    table = []

    def timed(o):
        try:
            run(o)
            ts = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                run(o)
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
        except ValueError as e:                       # an option set the launcher refuses (does not fit)
            table.append((dict(o), f'refused: {str(e)[:60]}'))
            return None
        if int(st[0].item()):
            raise RuntimeError('tensor-core level: a bounded wait ran out while tuning')
        ms = float(np.median(ts))
        table.append((dict(o), ms))
        return ms

    try:
        best = {}
        best_ms = timed(best)
        if best_ms is None:
            _LEVEL_CACHE[key] = None
            return None, table
        cand = _level_candidates(C, Lk)

        def consider(o):
            nonlocal best, best_ms
            ms = timed(o)
            if ms is not None and ms < best_ms:
                best, best_ms = dict(o), ms
        for k in cand['fir']:
            consider(dict(best, fir=k))
        for c in cand['copies']:
            consider(dict(best, copies=c))
        for c in cand['consumers']:
            consider(dict(best, consumers=c))
        for nt in cand['nt'][best.get('consumers', 8)]:
            consider(dict(best, nt=nt))
        if cand['repeat_off']:
            for nt in cand['nt16']:
                consider(dict(best, repeat=1, nt=nt))
        for sb in cand['sb']:
            consider(dict(best, sb=sb))
    finally:
        del x, ph, out, scr
        torch.cuda.empty_cache()
    _LEVEL_CACHE[key] = best
    if _cache_path():
        _save_cache(_cache_path())
    return best, table


def tune_levels(plan, reps=3):
    """tune_level for every level of a plan whose first pass can run on the tensor cores; the chosen options are
    stored in the plan's level records (key 'tc', read by DevicePlan) -> the list of per-level options (None for a
    level left to the other kernels)."""
    chosen = []
    Np = 1
    for lv in plan['levels']:
        opts = None
        if lv['C'] <= 64 and (lv['fir_k']['L'] if lv['fir_k'] is not None else 1) <= 96:
            opts, _ = tune_level(lv, Np, reps=reps)
        if opts is not None:
            lv['tc'] = dict(opts)
        chosen.append(opts)
        Np *= int(lv['C'])
    return chosen


def main():
    """python -m fastsar_b200.tune --workload spotlight_12k [--pmax 0.52] [--out path] [--reps 5]: time the launch
    options of the chosen form's tensor-core levels (precision float16, learned taps, 80 dB fallback filters, the
    given pmax) for a named workload's plan and write them, with whatever the cache already held, to `out` (default:
    the packaged file)."""
    import argparse
    from . import sim, learned
    ap = argparse.ArgumentParser()
    ap.add_argument('--workload', action='append', required=True)
    ap.add_argument('--out', default=PACKAGED_CACHE)
    ap.add_argument('--reps', type=int, default=5)
    ap.add_argument('--max-parents', type=int, default=4096)
    ap.add_argument('--pmax', type=float, default=0.52)
    a = ap.parse_args()
    _load_cache()
    taps = learned.LearnedTaps.load()
    for name in a.workload:
        w = sim.workload(name)
        col = w['col']
        T, _ = _plan.choose_T(col.ant, col.fmin + col.K * col.df, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'],
                              w['e2'], -40.0)
        pl = _plan.make_plan(col, w['nx'], w['ny'], w['spx'], w['spy'], T=T, nlev=3, pmax=a.pmax, atten=80.0,
                             e1=w['e1'], e2=w['e2'], taps=taps)
        Np = 1
        for i, lv in enumerate(pl['levels']):
            key = level_signature(lv, Np)
            _LEVEL_CACHE.pop(key, None)
            opts, table = tune_level(lv, Np, reps=a.reps, max_parents=a.max_parents)
            print(f'{name} level {i} {key}: {opts}')
            for o, ms in table:
                print(f'    {o}: {ms if isinstance(ms, str) else f"{ms:.3f} ms"}')
            Np *= int(lv['C'])
    _save_cache(a.out)
    print('wrote', a.out)


if __name__ == '__main__':
    main()
