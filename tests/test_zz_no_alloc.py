"""GPU test of ``dqb_mesolve_dense_noalloc``, the entry point for callers that cannot
allocate device memory -- for example code running inside a process whose framework has
already reserved nearly all of the GPU's memory for its own pool (JAX preallocates 75%
of it by default), where a cudaMalloc made on the library's behalf would fail or take
memory the framework does not track.  The entry point takes its scratch from a static
device array instead of a caller workspace.

It must give the same results as ``dqb_mesolve_dense`` (the workspace entry point) on
the same problem, on two calls in a row (the second call finds the first one's leftovers
in the shared array), with the tolerance the other GPU tests use: 1e-5 relative
Frobenius error per saved state and 1e-5 on expectation values.

This file is named so that pytest collects it last."""

import numpy as np
import pytest
import torch

from dynamiqs_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-5
NOALLOC_SCRATCH_BYTES = 8 << 20  # DQB_NOALLOC_SCRATCH_BYTES in include/dqb200.h


def _problem(batch, seed):
    w = workloads.batched_kerr(batch=batch, seed=seed)
    ts = np.linspace(0.0, 3.0, 16)
    dev = torch.device('cuda', 0)
    n, K = 64, 2
    bufs = dict(
        H=torch.from_numpy(np.ascontiguousarray(w['H'])).to(dev),
        L=torch.from_numpy(np.ascontiguousarray(np.stack(w['jump_ops'])[None])).to(dev),
        rho0=torch.from_numpy(np.ascontiguousarray(w['rho0'])).to(dev),
        E=torch.from_numpy(np.ascontiguousarray(np.stack(w['exp_ops']))).to(dev),
        ts=torch.from_numpy(ts).to(dev),
        zeros=torch.zeros(batch, dtype=torch.int32, device=dev),
    )
    prob = _lib.DenseProblem(
        n=n, n_jumps=K, n_exp=1, n_tsave=len(ts), batch=batch, H=bufs['H'].data_ptr(),
        L=bufs['L'].data_ptr(), rho0=bufs['rho0'].data_ptr(), rho0_is_ket=1,
        E=bufs['E'].data_ptr(), tsave=bufs['ts'].data_ptr(), H_index=None,
        L_index=bufs['zeros'].data_ptr(), rho0_index=bufs['zeros'].data_ptr())
    opts = _lib.OdeOptions(method=_lib.METHOD_TSIT5, form=_lib.FORM_HERMITIAN, rtol=1e-6,
                           atol=1e-8, safety=0.9, factormin=0.2, factormax=5.0,
                           max_steps=100_000, t0=0.0, save_states=1, check_hermitian=1)
    return prob, opts, bufs, len(ts)


def _outputs(batch, nt, n=64):
    dev = torch.device('cuda', 0)
    o = dict(states=torch.full((batch, nt, n, n), float('nan'), dtype=torch.complex64, device=dev),
             expects=torch.full((batch, 1, nt), float('nan'), dtype=torch.complex64, device=dev),
             infos=torch.full((batch, 3), -1, dtype=torch.int32, device=dev),
             status=torch.full((batch,), -1, dtype=torch.int32, device=dev))
    s = _lib.Outputs(states=o['states'].data_ptr(), expects=o['expects'].data_ptr(),
                     infos=o['infos'].data_ptr(), status=o['status'].data_ptr())
    return o, s


def _rel(x, ref):
    return (torch.linalg.norm((x - ref).reshape(*x.shape[:-2], -1), dim=-1)
            / torch.linalg.norm(ref.reshape(*ref.shape[:-2], -1), dim=-1)).max().item()


def test_noalloc_matches_workspace_entry_point(cuda_device):
    lib = _lib.load()
    batch = 40  # more instances than the 28 slots the static array holds at n = 64
    prob, opts, bufs, nt = _problem(batch, seed=3)
    stream = torch.cuda.current_stream().cuda_stream

    ref, ref_s = _outputs(batch, nt)
    ws_bytes = lib.dqb_mesolve_dense_workspace_size(64, 2, batch)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device='cuda')
    _lib.check(lib.dqb_mesolve_dense(prob, opts, ref_s, ws.data_ptr(), ws_bytes, stream),
               'dqb_mesolve_dense')
    torch.cuda.synchronize()
    assert int((ref['status'] != 0).sum()) == 0

    drops = []
    for call in range(4):
        got, got_s = _outputs(batch, nt)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _lib.check(lib.dqb_mesolve_dense_noalloc(prob, opts, got_s, stream),
                   'dqb_mesolve_dense_noalloc')
        torch.cuda.synchronize()
        drops.append(free_before - torch.cuda.mem_get_info()[0])
        if call >= 2:
            continue  # calls 2 and 3 only add samples of free memory
        assert int((got['status'] != 0).sum()) == 0
        assert _rel(got['states'], ref['states']) < TOL
        e_err = ((got['expects'] - ref['expects']).abs()
                 / ref['expects'].abs().clamp(min=1.0)).max().item()
        assert e_err < TOL
        assert torch.equal(got['infos'], ref['infos'])
    # Free device memory is a device-wide figure (other processes can move it), so the
    # check is coarse: the first call may reserve the static array when the driver loads
    # its module lazily (at most the array plus page rounding); no later call takes as
    # much as one instance slot (288 KiB at n = 64), so none allocates scratch.
    slot = 9 * 64 * 64 * 8
    assert drops[0] <= NOALLOC_SCRATCH_BYTES + (4 << 20), drops
    assert all(d < slot for d in drops[1:]), drops


def test_noalloc_rejects_sizes_beyond_its_kernel(cuda_device):
    lib = _lib.load()
    prob, opts, bufs, nt = _problem(2, seed=0)
    prob.n = 65
    _, s = _outputs(2, nt)
    assert lib.dqb_mesolve_dense_noalloc(prob, opts, s, None) == _lib.DQB_ERR_UNSUPPORTED
