"""Bounded waits: no tensor-core kernel spins for ever on an mbarrier.  The probe runs one
wait that nothing completes and must give up after its limit; the n <= 64 tensor-core
kernel, told that its waits give up at once, must end every instance it started with the
non-finite status, drain the MMAs it had issued, free its tensor memory and return -- and
the next launch in the same context must run normally.  Nothing here faults or hangs a
GPU: the failure is a host setting."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def test_probe_wait_gives_up_after_its_limit(cuda_device):
    lib = _lib.load()
    out = torch.zeros(2, dtype=torch.int32, device='cuda')
    _lib.check(lib.dqb_probe_bounded_wait(2_000_000, out.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream), 'probe')
    torch.cuda.synchronize()
    gave_up, waited_us = out.cpu().tolist()
    assert gave_up == 1
    assert 2_000 <= waited_us < 500_000
    assert lib.dqb_probe_bounded_wait(2_000_000_000, out.data_ptr(), None) == _lib.DQB_ERR_INVALID_ARGUMENT


def test_tensor_core_kernel_failure_path(cuda_device):
    lib = _lib.load()
    w = workloads.batched_kerr(batch=6, seed=1)
    ts = np.linspace(0.0, 0.5, 3)
    opts = dq.Options(precision='f16x3')
    ref = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=w['method'], options=opts)
    lib.dqb_set_tc_wait_limit_ns(1)
    try:
        with pytest.raises(RuntimeError, match='non-finite'):
            dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=w['method'], options=opts)
        torch.cuda.synchronize()  # the launch has returned: nothing is left spinning
    finally:
        lib.dqb_set_tc_wait_limit_ns(0)
    again = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=w['method'], options=opts)
    assert torch.equal(again.states, ref.states)
    assert torch.equal(again.infos.nsteps, ref.infos.nsteps)
