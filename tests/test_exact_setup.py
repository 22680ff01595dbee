"""ExactFormer's host-side set-up against the reference's (tests/golden/exact_setup.npz, made by the reference's
ExactFormer in float64): the tile, its predicted error, the tile centres, the per-pulse window of range bins and
the transform length, on geometries that pick 32 x 32 and 16 x 16 tiles. Runs on the CPU (the backend check is
bypassed: the set-up touches no GPU)."""
import numpy as np
import pytest


@pytest.mark.parametrize('case', ['r5k', 'r1k', 'wide'])
def test_exact_setup_matches_reference(golden, monkeypatch, case):
    from fastsar_b200 import api, exact
    monkeypatch.setattr(api, '_backend', lambda b: 'cuda')
    g = golden('exact_setup')
    fmin, df, K, nx, ny, spx, spy = g[f'{case}_scal']
    f = exact.ExactFormer(g[f'{case}_ant'], fmin, df, int(K), int(nx), int(ny), spx, spy)
    assert tuple(f.tile) == tuple(g[f'{case}_tile'])
    assert f.nfft == int(g[f'{case}_nfft'])
    assert f.W == int(g[f'{case}_W'])
    assert np.array_equal(np.asarray(f.blo, np.int64), g[f'{case}_blo'])
    np.testing.assert_allclose(f.cen, g[f'{case}_cen'], rtol=0, atol=1e-9)
    assert abs(f.predicted_error_db - float(g[f'{case}_err'])) < 1e-9
    assert f.inv_dr == pytest.approx(float(g[f'{case}_inv_dr']), rel=1e-15)
    assert f.kcyc == pytest.approx(float(g[f'{case}_kcyc']), rel=1e-15)


def test_exact_former_argument_errors(monkeypatch):
    from fastsar_b200 import api, exact, sim
    monkeypatch.setattr(api, '_backend', lambda b: 'cuda')
    col = sim.make_collect(res=0.5, scene=60.0, r0=5e3)
    with pytest.raises(ValueError, match='interp'):
        exact.ExactFormer(col.ant, col.fmin, col.df, col.K, 64, 64, 0.5, 0.5, interp='nearest')
    with pytest.raises(ValueError, match='float16-pair'):
        exact.ExactFormer(col.ant, col.fmin, col.df, col.K, 64, 64, 0.5, 0.5, profiles='float16-pair')
    with pytest.raises(ValueError, match='ref'):
        exact.ExactFormer(col.ant, col.fmin, col.df, col.K, 64, 64, 0.5, 0.5, ref=np.zeros(3))
    with pytest.raises(ValueError, match='range'):             # more range than c / (2 df) resolves
        exact.ExactFormer(col.ant, col.fmin, col.df, col.K, 4000, 64, 0.5, 0.5)
