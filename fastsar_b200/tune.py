"""The autotuner of a patch's plan: build a former for each candidate (levels, tile size, precision, taps, pmax),
drop those that cannot be built or formed or whose predicted final-stage error misses the target, time the rest on the patch's history
with CUDA events and keep the fastest. No counterpart in the reference, which plans every patch by fixed rules
(fastsar/patches.py:162-171 for the levels, fastsar/ffbp2.py:300-307 for the tile size).

    former, choice, table = tune_former(make, candidates, S_dev, target_db=-60.0)

make(**kwargs) -> ImageFormer; candidates: a list of kwargs; S_dev: the patch's history on the device.
"""
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
        except (ValueError, RuntimeError) as e:      # a shape a kernel refuses (FFBP_E_UNSUPPORTED), or an abort
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
