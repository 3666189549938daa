"""Failure paths of the scan, made to happen without faulting the GPU.

* Bounded device waits: a plan whose tensor-core waits get one mbarrier poll each makes
  the tensor-core y pass give up on its first wait (its operands cannot have landed
  yet). The kernel records the timeout, waits for its MMAs in flight, frees its tensor
  memory and returns; ``check`` raises TimeoutError (TM_E_TIMEOUT), the context stays
  usable, and the same plan with the default budget, and a fresh plan, match the oracle.
  The x and z passes of that plan run on the CUDA cores, so the only kernel whose waits
  run out is the y pass.
* Allocation failure injected on the host: a device-memory cap below what a plan needs
  makes plan creation fail with MemoryError before anything is allocated, as the
  reference surfaces allocation errors (tme/matching_exhaustive.py:122-141).
"""
import numpy as np
import pytest

from oracle import tm_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _case():
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(77)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    mask = syn.spherical_mask((12,) * 3, 6, center=(5.5,) * 3)
    target, _, _ = syn.make_tomogram((64, 512, 40), tmpl, 4, rng, scale=0.5)
    rots = syn.random_rotation_matrices(32, rng)
    return target, tmpl, mask, rots


def _plan(torch, target, tmpl, mask):
    from pytme_b200.matching import fourier_padding
    from pytme_b200.scores import ScanPlan

    _, fast, _, _ = fourier_padding(target.shape, tmpl.shape)
    plan = ScanPlan("FLCSphericalMask", fast, tmpl.shape, precision="mixed", batch=32)
    plan.set_xpass("fft")
    plan.set_zpass("fft")
    plan.set_ypass("tensor")
    plan.set_template(np.ascontiguousarray(tmpl[::-1, ::-1, ::-1]),
                      np.ascontiguousarray(mask[::-1, ::-1, ::-1]))
    tpad = torch.zeros(fast, dtype=torch.float32, device="cuda")
    tpad[tuple(slice(0, s) for s in target.shape)] = torch.as_tensor(target, device="cuda")
    plan.set_target(tpad)
    return plan, fast


def _run(torch, plan, fast, tmpl, rots, target):
    from pytme_b200.matching import fourier_padding, rigid_transform_matrices

    conv, fast2, _, shift = fourier_padding(target.shape, tmpl.shape)
    mats = torch.as_tensor(rigid_transform_matrices(rots, (np.asarray(tmpl.shape) - 1) / 2),
                           device="cuda")
    smax = torch.zeros(fast, dtype=torch.float32, device="cuda")
    sarg = torch.full(fast, -1, dtype=torch.int32, device="cuda")
    plan.run(mats, 0, smax, sarg)
    return smax, sarg, (conv, shift)


def _same_map(smax, sarg, geom, target, tmpl):
    conv, shift = geom
    return O.result_map(smax.cpu().numpy(), sarg.cpu().numpy(), shift, conv, target.shape,
                        tmpl.shape, "same")


def test_short_wait_budget_times_out_and_context_recovers(torch_cuda):
    torch = torch_cuda
    target, tmpl, mask, rots = _case()
    ref = O.scan(target, tmpl, rots, "FLCSphericalMask", template_mask=mask)
    plan, fast = _plan(torch, target, tmpl, mask)
    assert plan.ypass == "tensor"
    plan.set_wait_budget(1)
    _run(torch, plan, fast, tmpl, rots, target)
    with pytest.raises(TimeoutError):
        plan.check()
    # the flag was consumed: a second check passes
    plan.check()
    # same plan, default budget
    plan.set_wait_budget(0)
    smax, sarg, geom = _run(torch, plan, fast, tmpl, rots, target)
    plan.check()
    s, _ = _same_map(smax, sarg, geom, target, tmpl)
    tol = max(TOL, 2e-3 * float(np.sqrt(np.mean(np.square(ref["scores"], dtype=np.float64)))))
    assert np.abs(s - ref["scores"]).max() <= tol
    plan.close()
    # a fresh plan
    plan, fast = _plan(torch, target, tmpl, mask)
    smax, sarg, geom = _run(torch, plan, fast, tmpl, rots, target)
    plan.check()
    s, _ = _same_map(smax, sarg, geom, target, tmpl)
    assert np.abs(s - ref["scores"]).max() <= tol
    plan.close()


def test_device_memory_cap_surfaces_as_memory_error(torch_cuda):
    from pytme_b200 import _native as N
    from pytme_b200.scores import ScanPlan

    N.check(N.lib.tm_set_device_memory_limit(1 << 20))
    try:
        with pytest.raises(MemoryError, match="limit"):
            ScanPlan("FLCSphericalMask", (128, 128, 64), (16, 16, 16), precision="mixed",
                     batch=16)
    finally:
        N.check(N.lib.tm_set_device_memory_limit(0))
    plan = ScanPlan("FLCSphericalMask", (128, 128, 64), (16, 16, 16), precision="mixed", batch=16)
    assert plan.device_bytes > (1 << 20)
    plan.close()
