"""The range gate's plan (fastsar_b200.plan.gate_plan) against the reference's _gate_plan (tests/golden/gate.npz,
made by fastsar/api.py:272-300): the padding, the transform lengths and the samples kept exactly, the gated band's
first frequency and step to 1e-12, the taper to float32 rounding; on wide-band geometries (with and without a
reference range per pulse, a rectangular image) and a spotlight. Runs on the CPU."""
import numpy as np
import pytest


@pytest.mark.parametrize('case', ['wide', 'wide_ref', 'wide_rect', 'spot4k'])
def test_gate_plan_matches_reference(golden, case):
    from fastsar_b200 import plan
    g = golden('gate')
    fmin, df, K, nx, ny, spx, spy = g[f'{case}_scal']
    ref = g[f'{case}_ref'] if g[f'{case}_ref'].size else None
    e1, e2 = g[f'{case}_e']
    gp = plan.gate_plan(g[f'{case}_ant'], ref, fmin, df, int(K), int(nx), int(ny), spx, spy, e1, e2)
    assert [gp['npl'], gp['Kp'], gp['N'], gp['k0'], gp['k1']] == list(g[f'{case}_ints'])
    assert gp['fmin'] == pytest.approx(g[f'{case}_fl'][0], rel=1e-12)
    assert gp['df'] == pytest.approx(g[f'{case}_fl'][1], rel=1e-12)
    np.testing.assert_allclose(gp['taper'], g[f'{case}_taper'], rtol=1e-6, atol=1e-7)


def test_gate_taper():
    from fastsar_b200 import plan
    f = np.array([0.0, 1.0, 2.0, 3.0, 5.0, 6.0, 7.0])
    t = plan.taper(f, (2.0, 5.0), 1.0)
    np.testing.assert_allclose(t, [0.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0], atol=1e-12)
    assert plan.taper(np.array([1.5]), (2.0, 5.0), 1.0)[0] == pytest.approx(0.5)
