"""Test infrastructure: the CPU (NumPy, float64) oracle of the learned-tap network and its training step. Only
tests/ (and the fixture scripts) use it, as the checker of fastsar_b200/csrc/mlp.cu; nothing in the product calls it.

The network (no counterpart in the reference): an MLP 5 -> 64 -> 64 -> 64 -> 16 with GELU (x Phi(x), the exact
erf form) after each hidden layer. A query is one phase of one axis of a merge stage's decimation filter; its 16
outputs correct the 8 taps of that phase for the range axis (0..7) and the angle axis (8..15). Weights and hidden
activations are bfloat16 (rounded to nearest even, as the device kernels store them) and every sum is float64 here
(float32 on the device). The loss is mean |v - y|^2 over point-target pairs: v the decimated value of a target's
parent samples e^{2 pi i f t}, y its exact child value.
"""
import numpy as np
from scipy.special import erf

LAYERS = ((5, 64), (64, 64), (64, 64), (64, 16))


def bf16(x):
    """Round float values to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def init_params(seed=0):
    """He-style initial weights [(W [out, in], b [out]), ...] as float32."""
    rng = np.random.default_rng(seed)
    ps = []
    for i, o in LAYERS:
        ps.append((rng.standard_normal((o, i)).astype(np.float32) * np.float32(np.sqrt(2.0 / i)),
                   np.zeros(o, np.float32)))
    return ps


def forward(params, x, rounding=True):
    """x [B, 5] -> (taps [B, 16], cache). The weights and the hidden activations are rounded to bfloat16 (as on the
    device) unless rounding is False (the smooth network, for finite-difference checks of the gradient)."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    h = np.asarray(x, np.float64)
    cache = []
    for li, (W, b) in enumerate(params):
        Wb = rnd(W)
        z = h @ Wb.T + np.asarray(b, np.float64)
        cache.append((h, z, Wb))
        h = rnd(gelu(z)) if li < len(params) - 1 else z
    return h, cache


def phases(D):
    """Phase of each of the D taps groups in output samples: (q + 1/2) / D for even D, q / D for odd D."""
    return (np.arange(D) + (0.5 if D % 2 == 0 else 0.0)) / D


def tap_offsets(D):
    """[D, 8]: offset (output samples) of tap n of phase q, phi_q - 4 + n."""
    return phases(D)[:, None] - 4.0 + np.arange(8)[None, :]


def loss_and_grad(params, x, prior, scale, inst, weight, f, y, rounding=True):
    """The decimation loss of the learned taps and its gradients [(dW, db), ...] (float64): returns
    (sum weight |v - y|^2, grads of the mean). Instance i = (first query q0, D, axis) of inst [ninst, 3] uses the taps
    prior[q0 + q, n] + scale * out[q0 + q, 8 axis + n] at offsets tap_offsets(D)[q, n]; pair s of the instance
    (f [ninst, S] cycles per output sample, y [ninst, S] complex) decimates to v = (1 / D) sum_{q, n} tap
    e^{2 pi i f t}; the instance's pairs weigh weight[i] (None: 1). The rounding of the forward pass is passed
    straight through: the gradient is that of the smooth network evaluated at the rounded weights and
    activations."""
    out, cache = forward(params, x, rounding)
    ninst, S = f.shape
    dout = np.zeros_like(out)
    total = 0.0
    for i, (q0, D, ax) in enumerate(np.asarray(inst, np.int64)):
        taps = np.asarray(prior, np.float64)[q0:q0 + D] + scale * out[q0:q0 + D, 8 * ax:8 * ax + 8]
        X = np.exp(2j * np.pi * f[i][:, None, None] * tap_offsets(D)[None])          # [S, D, 8]
        v = np.einsum('sqn,qn->s', X, taps) / D
        e = v - y[i]
        wi = 1.0 if weight is None else float(weight[i])
        total += wi * float(np.sum(np.abs(e) ** 2))
        g = wi * np.real(np.conj(e)[:, None, None] * X).sum(0) * (2.0 / (ninst * S)) / D
        dout[q0:q0 + D, 8 * ax:8 * ax + 8] += scale * g
    d = dout
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        h, z, Wb = cache[li]
        if li < len(params) - 1:
            d = d * gelu_grad(z)
        grads[li] = (d.T @ h, d.sum(0))
        d = d @ Wb
    return total, grads


def adam_step(params, grads, state, lr, t, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on float32 master weights; state [(m_W, v_W, m_b, v_b), ...] updated in place."""
    out = []
    for (W, b), (dW, db), st in zip(params, grads, state):
        new = []
        for k, (p, gk) in enumerate(((W, dW), (b, db))):
            m, v = st[2 * k], st[2 * k + 1]
            m[...] = b1 * m + (1 - b1) * gk
            v[...] = b2 * v + (1 - b2) * gk * gk
            mh = m / (1 - b1 ** t)
            vh = v / (1 - b2 ** t)
            new.append((p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32))
        out.append(tuple(new))
    return out
