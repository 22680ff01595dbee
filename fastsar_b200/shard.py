"""One image formed on several GPUs, sharded by first-level child (the reference's first-level groups are independent
after the first level: fastsar/ffbp_cpu.py:278-291, fastsar/ffbp_cuda.py:1154-1198).

Each rank takes a contiguous range of the first level's children (child_ranges) and runs the same plan restricted to
them (restrict_plan): its share of every level's parents and of the final tiles, which cover disjoint pixels of the
image. A rank needs the whole history (one broadcast from the rank that holds it); its tiles are written into a
zeroed image, and the ranks' images are summed (the pixels are disjoint, so the sum is the assembly). With one rank
the plan is the whole plan.

    former = ShardedFormer(ant, fmin, df, K, nx, ny, spx, spy, e1, e2, precision=..., ...)   # torch.distributed set up
    img = former.form_device(S_dev, src=0)       # S_dev on rank src (others pass a buffer of the same shape or None)
"""
import numpy as np

from . import plan as _plan


def child_ranges(G, world):
    """Contiguous ranges [g0, g1) of G first-level children over `world` ranks, as even as possible (the first G %
    world ranks take one more)."""
    if world < 1:
        raise ValueError(f'world size must be positive, got {world}')
    base, extra = divmod(G, world)
    out, g0 = [], 0
    for r in range(world):
        g1 = g0 + base + (1 if r < extra else 0)
        out.append((g0, g1))
        g0 = g1
    return out


def restrict_plan(plan, g0, g1):
    """The plan restricted to first-level children g0 .. g1 - 1: every level's parent-indexed arrays and the final
    tiles sliced to the descendants of those children (the tile order nests each first-level child's tiles in one
    contiguous run), the first level's split recorded as (g1 - g0, 1). The restricted plan's tiles cover part of the
    padded grid ('partial': True)."""
    levels = plan['levels']
    G = levels[0]['C']
    if not 0 <= g0 < g1 <= G:
        raise ValueError(f'child range [{g0}, {g1}) outside the {G} first-level children')
    out = dict(plan)
    lv_out = []
    for l, lv in enumerate(levels):
        d = dict(lv)
        if l == 0:
            d['cen'] = np.ascontiguousarray(lv['cen'][:, g0:g1])
            d['sx'], d['sy'], d['C'] = g1 - g0, 1, g1 - g0
            d['d'] = np.ascontiguousarray(d['cen'][0] - lv['ref'][0])
        else:
            m = int(np.prod([v['C'] for v in levels[1:l]]))    # level l's parents per first-level child
            d['ref'] = np.ascontiguousarray(lv['ref'][g0 * m:g1 * m])
            d['cen'] = np.ascontiguousarray(lv['cen'][g0 * m:g1 * m])
        lv_out.append(d)
    tpc = int(np.prod([v['C'] for v in levels[1:]]))           # final tiles per first-level child
    fin = dict(plan['final'])
    fin['cen'] = np.ascontiguousarray(plan['final']['cen'][g0 * tpc:g1 * tpc])
    fin['first'] = np.ascontiguousarray(plan['final']['first'][g0 * tpc:g1 * tpc])
    out['levels'] = lv_out
    out['final'] = fin
    out['partial'] = True
    out['children'] = (g0, g1)
    return out


class ShardedFormer:
    """ImageFormer's plan on this rank's share of the first-level children. The ranks are torch.distributed's
    (one process per GPU, NCCL); without an initialised process group this rank forms the whole image. Arguments as
    ImageFormer's (aperture weights excepted). form_device(S_dev, src) broadcasts the history from rank src, forms
    this rank's tiles into a zeroed image and sums the ranks' images (all-reduce), so that every rank holds the
    image; the pixels of different ranks are disjoint, so the sum changes no value."""

    def __init__(self, ant, fmin, df, K, nx, ny, spx, spy, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), *, group=None,
                 **kw):
        import torch
        import torch.distributed as dist
        from .api import ImageFormer, DevicePlan, _final_mode
        if kw.get('aperture_weight') is not None:
            raise ValueError('ShardedFormer does not take aperture weights; form with ImageFormer')
        self.group = group
        self.dist = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if self.dist else 0
        self.world = dist.get_world_size(group) if self.dist else 1
        # the whole former plans once (its plan is the same on every rank); its device plan is replaced by the
        # rank's share
        whole = ImageFormer(ant, fmin, df, K, nx, ny, spx, spy, e1, e2, **kw)
        if whole.range_gate is not None:
            raise ValueError('ShardedFormer does not gate the history in range; form with ImageFormer')
        self.nx, self.ny, self.P, self.K = whole.nx, whole.ny, whole.P, whole.K
        G = whole._plan['levels'][0]['C']
        if self.world > G:
            raise ValueError(f'{self.world} ranks for {G} first-level children')
        self.children = child_ranges(G, self.world)[self.rank]
        sub = restrict_plan(whole._plan, *self.children)
        wp, wk = (whole.wp, whole.wk) if whole.window else (None, None)
        ref = kw.get('ref')
        self._dev = DevicePlan(sub, wp, wk, None, None if ref is None else np.asarray(ref, np.float64),
                               _final_mode(whole.precision), partial=True)
        self.T, self.levels, self.precision = whole.T, whole.levels, whole.precision
        del whole
        self._S = None

    def form_device(self, S_dev=None, src=0, out=None):
        """The image [nx, ny] complex64 on this rank's device: S_dev [P, K] complex64 on rank src (None elsewhere);
        broadcast, this rank's tiles formed, the ranks' images summed."""
        import torch
        import torch.distributed as dist
        dev = self._dev.device
        if self.dist and self.world > 1:
            if self.rank == src:
                S = S_dev.to(dev, torch.complex64).contiguous()
            else:
                if self._S is None:
                    self._S = torch.empty((self.P, self.K), dtype=torch.complex64, device=dev)
                S = self._S
            dist.broadcast(S, src, group=self.group)
        else:
            S = S_dev.to(dev, torch.complex64).contiguous()
        if out is None:
            out = torch.empty((self.nx, self.ny), dtype=torch.complex64, device=dev)
        out.zero_()
        self._dev.form(S, out)
        if self.dist and self.world > 1:
            dist.all_reduce(out, group=self.group)
        return out
