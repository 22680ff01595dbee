"""Failure reports of the tensor-core kernels, on a B200, without a GPU fault.

Every wait of the tensor-core pipelines (level pass 1, final stage) is bounded; one that runs out sets the block's
abort flag, the block winds down (no MMA left in flight, its tensor memory freed) and the plan's abort count rises.
The test hook ffbp_plan_test_wait makes the MMA issuers first wait, with a limit of a few milliseconds, on a barrier
that nothing completes: the wait runs out exactly as a stuck pipeline's would. The tests check that the failure is
reported whichever way the caller forms (check=False: by check() or by the next call; check=True: by the call
itself), that it is reported once, and that the plan then forms correct images again."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
if not torch.cuda.is_available():
    pytest.skip('no CUDA device', allow_module_level=True)


def _former(golden):
    from fastsar_b200 import ImageFormer, sim
    g = golden('image_spot512')
    w = sim.workload('spotlight_512')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, 512, 512, 0.25, 0.25, w['e1'], w['e2'], precision='float16')
    return f, torch.from_numpy(g['S']).cuda()


@pytest.mark.parametrize('kind', ['level_tc_gemm', 'final_tc'])
def test_bounded_wait_that_runs_out_is_reported(golden, kind):
    f, S = _former(golden)
    want = f.form_device(S).cpu().numpy()
    out = torch.empty((512, 512), dtype=torch.complex64, device='cuda')
    f._dev.test_wait(kind, 2000)
    # without check the call returns at once; the abort is raised by check(), once
    f.form_device(S, out, check=False)
    with pytest.raises(RuntimeError, match='bounded wait ran out'):
        f.check()
    f.check()
    # with check the call waits and raises its own abort
    with pytest.raises(RuntimeError, match='bounded wait ran out'):
        f.form_device(S, out)
    # an abort of a check=False call is raised by the plan's next call, before it launches anything
    f.form_device(S, out, check=False)
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match='earlier form call'):
        f.form_device(S, out, check=False)
    f.check()
    # the hook off: the same plan forms the same image as before, bit for bit
    f._dev.test_wait(None)
    got = f.form_device(S).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_batch_reports_an_abort(golden):
    """A batch's graph holds the launches as captured: captured with the hook on, every launch of it aborts, and
    each abort is reported (by the launch that waits, or by the next launch)."""
    from fastsar_b200 import BatchFormer
    f, S = _former(golden)
    f._dev.test_wait('final_tc', 2000)
    batch = BatchFormer([f])
    batch.histories[0].copy_(S)
    with pytest.raises(RuntimeError, match='image 0'):
        batch.form_device()
    batch.form_device(check=False)
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match='image 0'):
        batch.form_device(check=False)
    batch.check()
    del batch
    f._dev.test_wait(None)


def test_test_hook_rejects_bad_arguments(golden):
    from fastsar_b200 import _lib
    f, _ = _former(golden)
    L = _lib.load()
    with pytest.raises(ValueError, match='kind'):
        _lib.check(L.ffbp_plan_test_wait(f._dev.handle, 5, 100), 'ffbp_plan_test_wait')
    with pytest.raises(ValueError, match='limit'):
        _lib.check(L.ffbp_plan_test_wait(f._dev.handle, _lib.FFBP_KIND_FINAL_TC, 0), 'ffbp_plan_test_wait')


def test_transfer_that_did_not_deliver_is_reported(golden):
    """ffbp_form_host checks every upload with a sampled, position-weighted float64 sum computed on both sides of the
    transfer. The test hook ffbp_plan_test_transfer leaves one upload out (its device buffer keeps the history of
    two images before), as a transfer that did not deliver would: form_many raises naming that history; the hook is
    one call only, and the next call's images equal form_device's."""
    f, S = _former(golden)
    rng = np.random.default_rng(4)
    hs = [(golden('image_spot512')['S'] * (rng.standard_normal() + 1j * rng.standard_normal())).astype(np.complex64)
          for _ in range(3)]
    pinned = [torch.from_numpy(h).pin_memory() for h in hs]
    want = [f.form_device(torch.from_numpy(h).cuda()).cpu().numpy() for h in hs]
    f._dev.test_transfer(2)
    with pytest.raises(RuntimeError, match='history 2 did not reach the device'):
        f.form_many(pinned)
    got = f.form_many(pinned)
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


def test_workspace_that_does_not_fit_names_remedies():
    """A plan whose workspace exceeds the device (learned taps at pmax 0.95 on the 4,096-pulse spotlight: the
    Kaiser-sinc fallback's long filters and nearly no decimation ask for hundreds of GiB) raises MemoryError naming
    the sizes and the remedies, before any kernel runs, and leaves the device usable."""
    from fastsar_b200 import ImageFormer, sim
    w = sim.workload('spotlight_4k')
    col = w['col']
    f = ImageFormer(col.ant, col.fmin, col.df, col.K, w['nx'], w['ny'], w['spx'], w['spy'], w['e1'], w['e2'],
                    taps='learned', atten=80.0, pmax=0.95)
    S = torch.zeros((col.Np, col.K), dtype=torch.complex64, device='cuda')
    with pytest.raises(MemoryError, match='Remedies'):
        f.form_device(S)
    assert torch.zeros(4, device='cuda').sum().item() == 0.0
