"""Sharding one image by first-level child on a B200: the plans restricted to each rank's children (what each GPU of
a sharded formation runs) formed one after another on one GPU, their images summed, against the whole plan's image;
float32 and the tensor-core form. And ShardedFormer with one rank (no process group): the whole image."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


@pytest.mark.parametrize('precision', ['float32', 'float16'])
@pytest.mark.parametrize('world', [2, 3])
def test_shards_sum_to_the_whole_image(golden, precision, world):
    from fastsar_b200 import ImageFormer, sim, shard
    from fastsar_b200.api import DevicePlan, _final_mode
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision=precision)
    S = torch.from_numpy(g['S']).cuda()
    whole = f.form_device(S).cpu().numpy()
    total = torch.zeros((512, 512), dtype=torch.complex64, device='cuda')
    G = f._plan['levels'][0]['C']
    for g0, g1 in shard.child_ranges(G, world):
        sub = shard.restrict_plan(f._plan, g0, g1)
        dp = DevicePlan(sub, f.wp, f.wk, None, None, _final_mode(precision), partial=True)
        part = torch.zeros((512, 512), dtype=torch.complex64, device='cuda')
        dp.form(S, part)
        total += part
    got = total.cpu().numpy()
    d = np.abs(got - whole).max() / np.abs(whole).max()
    print(f'{precision}, {world} shards: max |difference| {d:.1e} of the peak, bitwise {np.array_equal(got, whole)}')
    assert d < 1e-6


def test_sharded_former_single_rank(golden):
    from fastsar_b200 import ImageFormer, sim, shard
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    args = (col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'])
    sf = shard.ShardedFormer(*args)
    assert sf.world == 1 and sf.children[0] == 0
    S = torch.from_numpy(g['S']).cuda()
    a = sf.form_device(S).cpu().numpy()
    b = ImageFormer(*args).form_device(S).cpu().numpy()
    assert np.array_equal(a, b)

