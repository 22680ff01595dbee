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
