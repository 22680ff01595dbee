"""The learned-tap network's CPU oracle (oracle/mlp_oracle.py) and the host side of fastsar_b200/learned.py, on the
CPU: the oracle's gradient against central differences of its own loss (on the smooth network, without the
bfloat16 rounding, which makes the loss piecewise constant), its Adam step, the bfloat16 rounding against torch's,
and the learned filters' layout (tap order, centre, margins) against the reference's decimator layout and a direct
decimation."""
import numpy as np
import pytest

import mlp_oracle as M


def _pairs(n_inst, S, seed):
    from fastsar_b200 import learned
    return learned.make_pairs(learned.instances(seed, n_inst), S, seed + 1)


def test_parameter_count_matches_the_library_layout():
    from fastsar_b200 import learned
    n = sum(o * i + o for i, o in M.LAYERS)
    assert n == learned.N_PARAMS == 9744
    assert learned.LAYERS == M.LAYERS
    ps = learned.unpack(np.arange(n, dtype=np.float32))
    assert [W.shape for W, _ in ps] == [(o, i) for i, o in M.LAYERS]
    assert ps[-1][1][-1] == n - 1


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.standard_normal(4096) * 10.0 ** rng.integers(-6, 6, 4096), [0.0, -0.0, 1.0, 3.0 / 256]])
    v = v.astype(np.float32)
    want = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(v), want)


@pytest.mark.parametrize('layer', [0, 1, 3])
def test_oracle_gradient_matches_central_differences(layer):
    from fastsar_b200 import learned
    params = M.init_params(seed=1)
    x, prior, inst, wt, f, y = _pairs(3, 16, seed=2)
    mean = lambda P: M.loss_and_grad(P, x, prior, learned.SCALE, inst, wt, f, y, rounding=False)[0] / f.size
    _, grads = M.loss_and_grad(params, x, prior, learned.SCALE, inst, wt, f, y, rounding=False)
    rng = np.random.default_rng(5)
    W, b = params[layer]
    h = 1e-3
    for _ in range(5):
        o, i = rng.integers(W.shape[0]), rng.integers(W.shape[1])
        for k, idx in ((0, (o, i)), (1, (o,))):
            plus = [[Wl.astype(np.float64).copy(), bl.astype(np.float64).copy()] for Wl, bl in params]
            minus = [[Wl.astype(np.float64).copy(), bl.astype(np.float64).copy()] for Wl, bl in params]
            plus[layer][k][idx] += h
            minus[layer][k][idx] -= h
            fd = (mean(plus) - mean(minus)) / (2 * h)
            an = grads[layer][k][idx]
            assert abs(fd - an) <= 1e-6 * max(1e-3, abs(an)) + 1e-9, (k, idx, fd, an)


def test_oracle_adam_step():
    from fastsar_b200 import learned
    params = M.init_params(seed=4)
    x, prior, inst, wt, f, y = _pairs(4, 32, seed=6)
    _, g = M.loss_and_grad(params, x, prior, learned.SCALE, inst, wt, f, y)
    state = [(np.zeros_like(W, np.float64), np.zeros_like(W, np.float64), np.zeros_like(b, np.float64),
              np.zeros_like(b, np.float64)) for W, b in params]
    new = M.adam_step(params, g, state, lr=1e-2, t=1)
    # the first Adam step moves every weight with a gradient well above eps by lr sign(g)
    for (W, b), (dW, db), (W1, b1) in zip(params, g, new):
        for p, gk, p1 in ((W, dW, W1), (b, db, b1)):
            nz = np.abs(gk) > 1e-4
            np.testing.assert_allclose((p - p1)[nz], (1e-2 * np.sign(gk))[nz], rtol=1e-3, atol=1e-6)


@pytest.mark.parametrize('D', [2, 3, 4, 7, 10, 21])
def test_learned_filter_layout_matches_the_reference_decimators(D):
    """The learned filter's (pl, pr, n_out, m) follow the reference's decimator layout (output j at input
    D (j - m) + (D - 1) / 2, out[j] = sum_r kern[r] x[D j + r - pl]): kern built from phase taps equal to the tap
    offsets decimates a ramp to the output positions; the prior's decimation of a constant is D."""
    from fastsar_b200 import learned, plan
    n_in = 200 + D
    pl, pr, n_out, m = learned.decimator_layout(n_in, D)
    assert n_out == plan.decimator_shape(n_in, D, 0.4, 10.0)[0] - 2 * plan.decimator_shape(n_in, D, 0.4, 10.0)[1] + 2 * m
    off = learned.kern_from_phases(learned.tap_offsets(D))          # kern[r] = offset of tap r in output samples
    r = np.arange(len(off))
    np.testing.assert_allclose(off * D, r - learned.centre(D), atol=1e-12)
    for j in (m, m + 3, n_out - m - 1):
        pos = D * (j - m) + (D - 1) / 2.0
        idx = D * j + r - pl
        np.testing.assert_allclose(idx - pos, off * D, atol=1e-12)
    assert pr == max(D * (n_out - 1) + len(off) - pl - n_in, 0)
    k = learned.kern_from_phases(learned.prior(D))
    x = np.ones(n_in + pl + pr + 8 * D)
    mid = n_out // 2
    assert abs(sum(k[t] * x[D * mid + t - pl + pl] for t in range(len(k))) / D - 1.0) < 1e-3


def test_prior_band_error_and_reference_kaiser():
    """The band-error metric on the reference's Kaiser-sinc decimators: longer filters (higher attenuation) have
    smaller errors, and the 8-output-sample prior sits near the 80 dB design."""
    from fastsar_b200 import learned, plan
    D, w = 7, 0.391
    e70 = learned.band_error_db(plan.decimator_fir(4096, D, w, 70.0)[0]['kern'], D, w)
    e80 = learned.band_error_db(plan.decimator_fir(4096, D, w, 80.0)[0]['kern'], D, w)
    ep = learned.band_error_db(learned.kern_from_phases(learned.prior(D)), D, w, learned.centre(D))
    assert e80 < e70 - 8.0
    assert abs(ep - e80) < 8.0
