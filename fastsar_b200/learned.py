"""Learned decimation taps (no counterpart in the reference): a small network that stands in for the fixed
Kaiser-sinc taps of the merge stages (fastsar/ffbp2.py:101-137, the `fir_k` range-axis and `fir_p` angle-axis
filters of every level).

A merge stage decimates each axis of its child data by D with pass fraction w: the child's band, |f| <= w / 2 in
cycles per output sample, must pass unchanged, and what would fold onto it, |f - n| <= w / 2 for integers n != 0,
must be stopped; the band between folds outside the child and is free. The reference meets this with a
Kaiser-windowed sinc whose length grows with its stop-band attenuation. Here the filter is 8 output samples wide
(8 D taps, the "8-tap" mode: 8 taps per phase) and its taps come from the network: one query per (stage, axis,
phase), features (phase, w, 1 / D, stage, axis), outputs corrections to the 8 taps of that phase on top of a
fixed Kaiser-sinc prior of the same width: tap = prior + SCALE * output.

Training pairs are point targets: a target at frequency f (its offset from the child's centre, in cycles per output
sample) leaves the parent samples e^{2 pi i f t} along the axis (exact along the frequency axis after the
re-centring on the child), and its exact child value is 1 inside the child's band and 0 where it would fold onto
it. Seeded random instances (D, w, stage, axis) each get S targets, half in the band and half in the folds; the
loss is the mean |v - y|^2 of the decimated values v. Forward, loss, backward and Adam are hand-written kernels
(fastsar_b200/csrc/mlp.cu, ffbp_mlp_*), their gradients checked against the CPU oracle (oracle/mlp_oracle.py);
training runs on the GPU: python -m fastsar_b200.learned train. The formers use the network through
`plan.make_plan(..., taps=LearnedTaps.load())`; a stage whose D or w the network was not trained for keeps the
Kaiser-sinc taps.
"""
import ctypes
import os

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL = os.path.join(HERE, 'data', 'learned_taps.npz')
N_PARAMS = 9744
LAYERS = ((5, 64), (64, 64), (64, 64), (64, 16))
WIDTH = 8                      # output samples spanned by the filter: 8 taps per phase
BETA = 7.0                     # Kaiser parameter of the prior
SCALE = 1.0 / 32.0             # output -> tap correction
D_RANGE = (2, 32)              # decimations and pass fractions the network is trained for
W_RANGE = (0.25, 0.65)


# --------------------------------------------------------------------------------------------- filter geometry
def phases(D):
    """Phase (output samples) of each of the D tap groups: (q + 1/2) / D for even D, q / D for odd D."""
    return (np.arange(D) + (0.5 if D % 2 == 0 else 0.0)) / D


def tap_offsets(D):
    """[D, 8]: offset (output samples) of tap n of phase q from the output sample, phi_q - 4 + n."""
    return phases(D)[:, None] - WIDTH / 2 + np.arange(WIDTH)[None, :]


def prior(D):
    """[D, 8] float64: the Kaiser-windowed sinc (cut-off half the output rate, beta BETA, half width 4 output
    samples) at tap_offsets(D); D times its sum is about D (the reference's decimators sum D inputs per output)."""
    t = tap_offsets(D)
    x = np.clip(1.0 - (t / (WIDTH / 2)) ** 2, 0.0, 1.0)
    return np.sinc(t) * np.i0(BETA * np.sqrt(x)) / np.i0(BETA)


def features(D, w, stage, axis):
    """[D, 5] float32 query rows of one (stage, axis) filter: the phase, the pass fraction w, 1 / D, the stage and
    the axis, each mapped onto about [-1, 1] over the trained ranges."""
    wc, wh = (W_RANGE[0] + W_RANGE[1]) / 2, (W_RANGE[1] - W_RANGE[0]) / 2
    return np.stack([2.0 * phases(D) - 1.0, np.full(D, (w - wc) / wh), np.full(D, 4.0 / D - 1.0),
                     np.full(D, stage / 1.5 - 1.0), np.full(D, 2.0 * axis - 1.0)], 1).astype(np.float32)


def kern_from_phases(taps):
    """[D, 8] taps by (phase q, tap n) -> the FIR kernel of 8 D taps in input order: kern[n D + q] = taps[q, n]."""
    return np.ascontiguousarray(np.asarray(taps).T.reshape(-1))


def decimator_layout(n_in, D):
    """(pl, pr, n_out, m) of an 8-output-sample filter: output j sits at input D (j - m) + (D - 1) / 2 with margin
    m = 4, and out[j] = sum_r kern[r] x[D j + r - pl] (the layout of the reference's decimators,
    fastsar/ffbp2.py:72-137)."""
    m = WIDTH // 2
    c2 = 2 * (WIDTH // 2) * D - (1 if D % 2 == 0 else 0)        # twice the centre tap's index
    pl = (2 * D * m - (D - 1) + c2) // 2
    n_out = -(-int(n_in) // D) + 2 * m
    L = WIDTH * D
    pr = max(D * (n_out - 1) + L - pl - int(n_in), 0)
    return pl, pr, n_out, m


def centre(D):
    """Index of the learned kernel's centre tap (input samples): its taps run from -4 D + 1/2 to 4 D - 1/2 about
    the output sample for even D, from -4 D to 4 D - 1 for odd D."""
    return (WIDTH * D - 1) / 2.0 if D % 2 == 0 else WIDTH * D / 2.0


def band_error_db(kern, D, w, c=None, n=4001):
    """Mean |v - y|^2 (dB) of a decimation kernel over the child's band and its folds, on a uniform grid of n
    frequencies per band; kern in input order with its centre at index c (default (len - 1) / 2, the reference's
    symmetric kernels)."""
    L = len(kern)
    t = (np.arange(L) - ((L - 1) / 2.0 if c is None else c)) / D
    u = np.linspace(-w / 2, w / 2, n)
    err, cnt = 0.0, 0
    for k in range(-(D // 2), D // 2 + 1):
        f = u + k
        f = f[np.abs(f) <= D / 2]
        v = np.exp(2j * np.pi * np.outer(f, t)) @ np.asarray(kern, np.float64) / D
        err += np.sum(np.abs(v - (1.0 if k == 0 else 0.0)) ** 2)
        cnt += len(f)
    return float(10 * np.log10(err / cnt))


# --------------------------------------------------------------------------------------------- the network
class LearnedTaps:
    """The network's parameters (float32, per layer W [out, in] then b [out]) and its GPU kernels. The last layer
    starts at zero, so that an untrained network gives the prior's taps."""

    def __init__(self, params=None, seed=0):
        if params is None:
            rng = np.random.default_rng(seed)
            parts = []
            for li, (i, o) in enumerate(LAYERS):
                W = rng.standard_normal((o, i)) * np.sqrt(2.0 / i)
                if li == len(LAYERS) - 1:
                    W = np.zeros((o, i))
                parts += [W.astype(np.float32).ravel(), np.zeros(o, np.float32)]
            params = np.concatenate(parts)
        self.params = np.ascontiguousarray(params, np.float32)
        if self.params.size != N_PARAMS:
            raise ValueError(f'the network has {N_PARAMS} parameters, got {self.params.size}')
        self._cache = {}

    @property
    def ident(self):
        """A short name of these parameters (for plan signatures)."""
        import hashlib
        return 'learned:' + hashlib.sha1(self.params.tobytes()).hexdigest()[:12]

    @classmethod
    def load(cls, path=MODEL):
        with np.load(path) as z:
            return cls(z['params'])

    def save(self, path=MODEL, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params, **{k: np.asarray(v) for k, v in meta.items()})

    def outputs(self, x):
        """x [nq, 5] query rows -> outputs [nq, 16] (float32) by the inference kernel."""
        import torch
        L = _lib.load()
        dev = torch.device('cuda', torch.cuda.current_device())
        xd = torch.as_tensor(np.ascontiguousarray(x, np.float32)).to(dev)
        p = torch.from_numpy(self.params).to(dev)
        nq = xd.shape[0]
        out = torch.empty((nq, 16), dtype=torch.float32, device=dev)
        work = torch.empty(int(L.ffbp_mlp_work_bytes(nq)) // 4 + 16, dtype=torch.float32, device=dev)
        _lib.check(L.ffbp_mlp_taps(p.data_ptr(), xd.data_ptr(), nq, out.data_ptr(), work.data_ptr(),
                                   torch.cuda.current_stream(dev).cuda_stream), 'ffbp_mlp_taps')
        return out.cpu().numpy()

    def phase_taps(self, D, w, stage, axis):
        """[D, 8] float64 taps (by phase and tap) of the (stage, axis) filter of decimation D and pass fraction w."""
        key = (int(D), float(w), int(stage), int(axis))
        if key not in self._cache:
            out = self.outputs(features(D, w, stage, axis))[:, 8 * axis:8 * axis + 8].astype(np.float64)
            self._cache[key] = prior(D) + SCALE * out
        return self._cache[key]

    def covers(self, D, w):
        return D_RANGE[0] <= D <= D_RANGE[1] and W_RANGE[0] <= w <= W_RANGE[1]

    def decimator(self, n_in, D, pass_frac, stage, axis):
        """The learned decimator of n_in samples by D in the layout of plan.decimator_fir: (dict(kern, pl, pr,
        n_out, L), m), or None where the network does not cover (D, pass_frac)."""
        if not self.covers(D, pass_frac):
            return None
        kern = kern_from_phases(self.phase_taps(D, pass_frac, stage, axis))
        kern.flags.writeable = False
        pl, pr, n_out, m = decimator_layout(n_in, D)
        return dict(kern=kern, pl=pl, pr=pr, n_out=n_out, L=len(kern)), m

    def _device_pairs(self, pairs):
        import torch
        dev = torch.device('cuda', torch.cuda.current_device())
        x, prior_, inst, wt, f, y = pairs
        return (torch.as_tensor(np.ascontiguousarray(x, np.float32)).to(dev),
                torch.as_tensor(np.ascontiguousarray(prior_, np.float32)).to(dev),
                torch.as_tensor(np.ascontiguousarray(inst, np.int32)).to(dev),
                torch.as_tensor(np.ascontiguousarray(wt, np.float32)).to(dev),
                torch.as_tensor(np.ascontiguousarray(f, np.float64)).to(dev),
                torch.as_tensor(np.ascontiguousarray(y, np.complex64)).to(dev))

    def grad(self, pairs):
        """(sum |v - y|^2, gradient of the mean) over the pairs by the device kernels (the gradient check)."""
        import torch
        L = _lib.load()
        dev = torch.device('cuda', torch.cuda.current_device())
        x, pr, inst, wt, f, y = self._device_pairs(pairs)
        p = torch.from_numpy(self.params).to(dev)
        nq, (ninst, S) = x.shape[0], f.shape
        grad = torch.empty(N_PARAMS, dtype=torch.float32, device=dev)
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
        work = torch.empty(int(L.ffbp_mlp_work_bytes(nq)) // 4 + 16, dtype=torch.float32, device=dev)
        _lib.check(L.ffbp_mlp_grad(p.data_ptr(), x.data_ptr(), nq, pr.data_ptr(), ctypes.c_float(SCALE), inst.data_ptr(),
                                   wt.data_ptr(), ninst, f.data_ptr(), y.data_ptr(), S, grad.data_ptr(), loss.data_ptr(),
                                   work.data_ptr(), torch.cuda.current_stream(dev).cuda_stream), 'ffbp_mlp_grad')
        return float(loss.item()), grad.cpu().numpy()

    def train(self, pairs, steps=60000, lr=3e-3, lr_end=3e-6, log=None, every=5000):
        """Adam over all pairs each step (full batch), the learning rate decaying geometrically from lr to lr_end.
        Returns [(step, mean loss)] every `every` steps."""
        import torch
        L = _lib.load()
        dev = torch.device('cuda', torch.cuda.current_device())
        x, pr, inst, wt, f, y = self._device_pairs(pairs)
        nq, (ninst, S) = x.shape[0], f.shape
        p = torch.from_numpy(self.params.copy()).to(dev)
        adam = torch.zeros(2 * N_PARAMS, dtype=torch.float32, device=dev)
        work = torch.empty(int(L.ffbp_mlp_work_bytes(nq)) // 4 + 16, dtype=torch.float32, device=dev)
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
        s = torch.cuda.current_stream(dev).cuda_stream
        hist = []
        for t in range(1, steps + 1):
            rate = lr * (lr_end / lr) ** ((t - 1) / max(1, steps - 1))
            _lib.check(L.ffbp_mlp_train_step(p.data_ptr(), adam.data_ptr(), x.data_ptr(), nq, pr.data_ptr(),
                                             ctypes.c_float(SCALE), inst.data_ptr(), wt.data_ptr(), ninst, f.data_ptr(),
                                             y.data_ptr(),
                                             S, ctypes.c_float(rate), t, loss.data_ptr(), work.data_ptr(), s),
                       'ffbp_mlp_train_step')
            if t % every == 0 or t == 1 or t == steps:
                hist.append((t, float(loss.item()) / (ninst * S)))
                if log:
                    log(f'step {t}: loss {10 * np.log10(hist[-1][1]):.2f} dB')
        self.params = p.cpu().numpy()
        self._cache = {}
        return hist


def unpack(params):
    """Flat parameters -> [(W [out, in], b [out]), ...]."""
    out, o = [], 0
    for i, n in LAYERS:
        W = params[o:o + n * i].reshape(n, i)
        o += n * i
        out.append((W, params[o:o + n]))
        o += n
    return out


# --------------------------------------------------------------------------------------------- the pairs
def instances(seed, n):
    """n seeded random (D, w, stage, axis) filter instances over the trained ranges."""
    rng = np.random.default_rng(seed)
    D = rng.integers(D_RANGE[0], D_RANGE[1] + 1, n)
    w = rng.uniform(W_RANGE[0], W_RANGE[1], n)
    return [(int(d), float(v), int(st), int(ax)) for d, v, st, ax in
            zip(D, w, rng.integers(0, 4, n), rng.integers(0, 2, n))]


def make_pairs(insts, S, seed):
    """Training pairs of filter instances: (x [nq, 5], prior [nq, 8], inst [ninst, 3], weight [ninst], f [ninst, S],
    y [ninst, S]). Per instance S point targets: the first half in the child's band (child value 1), the rest
    spread over the folds onto it inside the input band (child value 0). An instance weighs the inverse of the
    prior's loss on its pairs (normalised to a mean of 1), so that narrow and wide bands count alike."""
    rng = np.random.default_rng(seed)
    xs, ps, inst = [], [], []
    f = np.empty((len(insts), S))
    y = np.zeros((len(insts), S), np.complex64)
    q0 = 0
    for i, (D, w, st, ax) in enumerate(insts):
        xs.append(features(D, w, st, ax))
        ps.append(prior(D))
        inst.append((q0, D, ax))
        q0 += D
        h = S // 2
        f[i, :h] = rng.uniform(-w / 2, w / 2, h)
        y[i, :h] = 1.0
        folds = np.array([k for k in range(-(D // 2), D // 2 + 1) if k != 0], np.float64)
        g = folds[rng.integers(0, len(folds), S - h)] + rng.uniform(-w / 2, w / 2, S - h)
        f[i, h:] = np.clip(g, -D / 2, D / 2)
    wt = np.empty(len(insts))
    for i, (D, w, st, ax) in enumerate(insts):
        v = np.exp(2j * np.pi * f[i][:, None, None] * tap_offsets(D)[None]).reshape(S, -1) @ prior(D).ravel() / D
        wt[i] = 1.0 / max(np.mean(np.abs(v - y[i]) ** 2), 1e-30)
    wt /= wt.mean()
    return (np.concatenate(xs), np.concatenate(ps).astype(np.float32), np.asarray(inst, np.int32),
            wt.astype(np.float32), f, y)


def kaiser_of_length(D, w, L):
    """The reference's Kaiser-sinc decimator (fastsar/ffbp2.py:101-137) with the highest stop-band attenuation
    (0.25 dB steps) whose kernel has at most L taps."""
    from .plan import decimator_fir
    lo, hi = 20.0, 200.0
    while hi - lo > 0.25:
        mid = 0.5 * (lo + hi)
        if decimator_fir(4096, D, w, mid)[0]['L'] <= L:
            lo = mid
        else:
            hi = mid
    return decimator_fir(4096, D, w, lo)[0]['kern']


def evaluate(model, insts, atten=80.0):
    """Per instance the band error (dB) of the learned taps, the prior alone, the reference's Kaiser-sinc decimator
    of no more taps than the learned filter (kaiser_same) and the one at `atten` (kaiser, with its length in
    taps): a list of dicts."""
    from .plan import decimator_fir
    rows = []
    for D, w, st, ax in insts:
        k = kern_from_phases(model.phase_taps(D, w, st, ax))
        kp = kern_from_phases(prior(D))
        kr = decimator_fir(4096, D, w, atten)[0]['kern']
        ks = kaiser_of_length(D, w, len(k))
        rows.append(dict(D=D, w=w, stage=st, axis=ax, learned=band_error_db(k, D, w, centre(D)),
                         prior=band_error_db(kp, D, w, centre(D)), kaiser_same=band_error_db(ks, D, w),
                         kaiser=band_error_db(kr, D, w), taps=len(k), kaiser_taps=len(kr)))
    return rows


def main(argv=None):
    import argparse
    import time
    ap = argparse.ArgumentParser(description='train the learned decimation taps on the GPU')
    ap.add_argument('cmd', choices=('train', 'eval'))
    ap.add_argument('--instances', type=int, default=8192)
    ap.add_argument('--pairs', type=int, default=256, help='point targets per instance')
    ap.add_argument('--steps', type=int, default=60000)
    ap.add_argument('--lr', type=float, default=3e-3)
    ap.add_argument('--lr-end', type=float, default=3e-6)
    ap.add_argument('--out', default=MODEL)
    args = ap.parse_args(argv)
    if args.cmd == 'train':
        t0 = time.time()
        pairs = make_pairs(instances(1, args.instances), args.pairs, seed=2)
        m = LearnedTaps(seed=0)
        hist = m.train(pairs, steps=args.steps, lr=args.lr, lr_end=args.lr_end, log=lambda s: print(s, flush=True),
                       every=max(1, args.steps // 12))
        print(f'trained in {time.time() - t0:.0f} s', flush=True)
        m.save(args.out, loss_db=10 * np.log10(np.array(hist)[:, 1]), steps=args.steps, lr=args.lr, lr_end=args.lr_end,
               instances=args.instances, pairs=args.pairs)
    m = LearnedTaps.load(args.out)
    rows = evaluate(m, instances(10 ** 6, 64))
    for key in ('learned', 'prior', 'kaiser_same', 'kaiser'):
        print(key, round(float(np.mean([r[key] for r in rows])), 2), 'dB')
    print('taps', np.mean([r['taps'] for r in rows]), 'kaiser 80 dB taps', np.mean([r['kaiser_taps'] for r in rows]))


if __name__ == '__main__':
    main()
