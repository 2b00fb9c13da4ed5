"""GPU parity of the sparse-DIA path (``dqb_lindblad_rhs_dia``, ``dqb_mesolve_dia``)
against the oracle's DIA restatement (``oracle.lindblad``, following
dynamiqs/qarrays/sparsedia_primitives.py) and against the dense kernel.

Solves are held to the bar of tests/parity.py; single right-hand sides are compared at
2e-6 relative."""

import ctypes

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib, workloads
from dynamiqs_b200.qarrays import SparseDIA
from oracle import lindblad as lb
from oracle.mesolve import mesolve as oracle_mesolve
from tests.parity import assert_solve_parity

pytestmark = pytest.mark.gpu


def rel_frob(x, ref):
    return np.linalg.norm(np.asarray(x) - ref, axis=(-2, -1)) / np.maximum(
        np.linalg.norm(ref, axis=(-2, -1)), 1e-30)


def _rand_dia(n, offsets, rng):
    d = (rng.normal(size=(len(offsets), n)) + 1j * rng.normal(size=(len(offsets), n))) / np.sqrt(n)
    for i, k in enumerate(offsets):
        if k >= 0:
            d[i, :k] = 0
        else:
            d[i, n + k:] = 0
    return SparseDIA(offsets, d.astype(np.complex64))


def _problem_struct(H, Ls, n, batch):
    c64 = torch.complex64
    h_off = (ctypes.c_int32 * len(H.offsets))(*H.offsets)
    l_nd = (ctypes.c_int32 * max(len(Ls), 1))(*[len(L.offsets) for L in Ls])
    lo = [k for L in Ls for k in L.offsets]
    l_off = (ctypes.c_int32 * max(len(lo), 1))(*lo)
    H_d = torch.from_numpy(np.ascontiguousarray(H.diags)).to('cuda', c64)
    L_d = torch.from_numpy(np.ascontiguousarray(np.concatenate([L.diags for L in Ls], axis=-2))).to('cuda', c64)
    p = _lib.DiaProblem(n=n, n_jumps=len(Ls), batch=batch, h_ndiag=len(H.offsets),
                        h_offsets=ctypes.cast(h_off, ctypes.c_void_p), h_diags=H_d.data_ptr(),
                        l_ndiag=ctypes.cast(l_nd, ctypes.c_void_p),
                        l_offsets=ctypes.cast(l_off, ctypes.c_void_p), l_diags=L_d.data_ptr())
    return p, [h_off, l_nd, l_off, H_d, L_d]


@pytest.mark.parametrize('tile', [0, 8, 108, 116, 208, 316, 408, 508, 604, 608, 708])
@pytest.mark.parametrize('form', [_lib.FORM_HERMITIAN, _lib.FORM_STANDARD])
@pytest.mark.parametrize('n', [10, 77, 300])
def test_rhs_dia_matches_oracle(cuda_device, form, n, tile):
    """Every stencil kernel (generic; tiled, 8 rows; staged, 8 and 16 rows) against the
    oracle, on operators whose offsets make the edges and the shared-memory groups ragged."""
    rng = np.random.default_rng(n)
    B = 2
    Hs = [_rand_dia(n, (-2, 0, 2), rng) for _ in range(B)]
    H = SparseDIA((-2, 0, 2), np.stack([h.diags for h in Hs]))
    H = SparseDIA(H.offsets, 0.5 * (H.diags + np.stack([h.dag().diags[[2, 1, 0]] for h in Hs])))
    Ls = [_rand_dia(n, (-2, -1, 1, 3), rng), _rand_dia(n, (1,), rng)]
    Ls = [SparseDIA(L.offsets, np.stack([L.diags] * B)) for L in Ls]
    Y = (rng.normal(size=(B, n, n)) + 1j * rng.normal(size=(B, n, n))) / n
    rho = Y @ np.conj(np.swapaxes(Y, -1, -2))
    if form == _lib.FORM_STANDARD:
        rho = rho + 0.1 * Y
    rho = rho.astype(np.complex64)
    p, keep = _problem_struct(H, Ls, n, B)
    r_d = torch.from_numpy(np.ascontiguousarray(rho)).to('cuda')
    out = torch.empty_like(r_d)
    ws = torch.empty(1 << 20, dtype=torch.uint8, device='cuda')
    lib = _lib.load()
    _lib.check(lib.dqb_lindblad_rhs_dia_tiled(p, form, tile, r_d.data_ptr(), out.data_ptr(),
                                              ws.data_ptr(), ws.numel(),
                                              torch.cuda.current_stream().cuda_stream), 'rhs_dia')
    got = out.cpu().numpy()
    for b in range(B):
        Hb = (H.offsets, H.diags[b].astype(complex))
        Lb = [(L.offsets, L.diags[b].astype(complex)) for L in Ls]
        if form == _lib.FORM_HERMITIAN:
            ref = lb.vf_hermitian_dia(Hb, Lb, rho[b].astype(complex))
        else:
            ref = lb.vf_standard(lb.dia_to_dense(*Hb), [lb.dia_to_dense(*x) for x in Lb],
                                 rho[b].astype(complex))
        assert rel_frob(got[b], ref) < 2e-6


def _oracle_compare(res, w, b, method='Tsit5'):
    H = (w['H'].offsets, w['H'].diags[b])
    Ls = [(L.offsets, L.diags) for L in w['jump_ops']]
    m = w['method']
    return assert_solve_parity(res.states[b].cpu().numpy(), None, int(res.infos.nsteps[b]), H,
                               Ls, w['rho0'], w['tsave'], None, method, m.rtol, m.atol)


def test_coupled_kerr_dia_small_vs_oracle(cuda_device):
    """Two coupled Kerr modes of 10 levels (n = 100 > 64: the DIA stepper path)."""
    w = workloads.coupled_kerr_dia(batch=2, m=10, seed=5)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], method=w['method'])
    assert res.states.shape == (2, 11, 100, 100)
    assert int((res.infos.nsteps > 0).sum()) == 2
    for b in range(2):
        _oracle_compare(res, w, b)


@pytest.mark.parametrize('tile', [1, 8, 208, 216, 308, 316, 408, 508, 608, 708])
@pytest.mark.parametrize('m', [10, 18])
def test_dia_solve_every_stencil_shape_vs_oracle(cuda_device, m, tile):
    """The DIA solve with the stencil shape forced, hermitian form: the wide shapes
    (2xx-5xx) write the stage slots on the upper 32 x 32 tiles only (no mirror), the
    others the whole matrix.  n = 100 and 324 (not multiples of the 32-row tiles or of the
    CTA's column band) against the oracle, and every shape's states and expectation values
    against the generic kernel's within the tolerance."""
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    w = workloads.coupled_kerr_dia(batch=2, m=m, seed=5)
    E = [np.diag(np.arange(m * m)).astype(np.complex64)]
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                  options=dq.Options(), H=w['H'], Ls=w['jump_ops'], Es=E, plan=plan)
    prep = integ._prepare_dia(_lib.load())
    integ._tuned['tile'] = tile
    res = prep.launch().result()
    for b in range(2):
        _oracle_compare(res, w, b)
    st = res.states.cpu().numpy().copy()  # (the next launch reuses the output buffers)
    ex = res.expects.cpu().numpy().copy()
    assert np.abs(st - np.conj(np.swapaxes(st, -1, -2))).max() < 1e-6
    if m == 10:
        integ._tuned['tile'] = 1
        ref = prep.launch().result()
        assert rel_frob(st, ref.states.cpu().numpy()).max() < w['method'].rtol
        np.testing.assert_allclose(ex, ref.expects.cpu().numpy(), rtol=w['method'].rtol, atol=1e-6)


def test_dia_path_equals_dense_kernel_at_n64(cuda_device):
    """Same problem through dqb_mesolve_dia and dqb_mesolve_dense (n = 64)."""
    w = workloads.coupled_kerr_dia(batch=3, m=8, seed=2)
    integ_dense = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], method=w['method'])
    # force the DIA path through the integrator's DIA runner
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                  options=dq.Options(), H=w['H'], Ls=w['jump_ops'], Es=None, plan=plan)
    res_dia = integ._run_dia(_lib.load())
    dn = np.abs(res_dia.infos.nsteps.cpu().numpy() - integ_dense.infos.nsteps.cpu().numpy())
    assert dn.max() <= 1
    assert rel_frob(res_dia.states.cpu().numpy(), integ_dense.states.cpu().numpy()).max() < 1e-5


def test_dia_expects_save_states_false_and_standard_form(cuda_device):
    w = workloads.coupled_kerr_dia(batch=1, m=9, seed=4)
    n = 81
    E = [np.diag(np.arange(n)).astype(np.complex64)]
    full = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=E, method=w['method'])
    last = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=E, method=w['method'],
                      options=dq.Options(save_states=False))
    std = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=E, method=w['method'],
                     options=dq.Options(assume_hermitian=False))
    assert last.states.shape == (1, 1, n, n)
    assert rel_frob(last.states[:, 0].cpu().numpy(), full.states[:, -1].cpu().numpy()).max() < 1e-5
    ref_e = np.einsum('ij,tji->t', E[0], full.states[0].cpu().numpy().astype(complex))
    np.testing.assert_allclose(full.expects[0, 0].cpu().numpy(), ref_e, rtol=1e-5, atol=1e-5)
    assert rel_frob(std.states.cpu().numpy(), full.states.cpu().numpy()).max() < 1e-5
    np.testing.assert_allclose(std.expects.cpu().numpy(), full.expects.cpu().numpy(), rtol=1e-5, atol=1e-5)


@pytest.fixture(scope='module')
def coupled_kerr_4096_rhs():
    """Coupled-Kerr operators at their full size (two 64-level modes, n = 4096; H offsets
    {-64, -63, 0, 63, 64}, jumps {+64} and {+1}), a random hermitian X and the oracle's
    hermitian right-hand side of it in complex128."""
    w = workloads.coupled_kerr_dia(batch=1, m=64, seed=0)
    n = 4096
    rng = np.random.default_rng(4096)
    Y = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / (2 * n)
    X = (Y + np.conj(Y.T)).astype(np.complex64)
    Hb = (w['H'].offsets, w['H'].diags[0].astype(complex))
    Lb = [(L.offsets, L.diags.astype(complex)) for L in w['jump_ops']]
    ref = lb.vf_hermitian_dia(Hb, Lb, X.astype(complex))
    return w, X, ref


@pytest.mark.parametrize('tile', [0, 4, 8, 16, 108, 116, 208, 216, 308, 316, 408, 508, 604, 608, 708])
def test_rhs_dia_full_size_every_stencil(cuda_device, coupled_kerr_4096_rhs, tile):
    """One right-hand side at n = 4096 with the workload's own offsets (+-63/+-64 select
    other row groups in the staged kernel and other halos in the tiled one than the small
    cases above) through every stencil shape, against the oracle at 2e-6."""
    w, X, ref = coupled_kerr_4096_rhs
    n = 4096
    Ls = [SparseDIA(L.offsets, L.diags[None]) for L in w['jump_ops']]
    p, keep = _problem_struct(w['H'], Ls, n, 1)
    r_d = torch.from_numpy(np.ascontiguousarray(X[None])).to('cuda')
    out = torch.empty_like(r_d)
    ws = torch.empty(1 << 20, dtype=torch.uint8, device='cuda')
    lib = _lib.load()
    _lib.check(lib.dqb_lindblad_rhs_dia_tiled(p, _lib.FORM_HERMITIAN, tile, r_d.data_ptr(),
                                              out.data_ptr(), ws.data_ptr(), ws.numel(),
                                              torch.cuda.current_stream().cuda_stream), 'rhs_dia')
    got = out[0].cpu().numpy()
    assert rel_frob(got, ref) < 2e-6
    if tile >= 200:
        # the wide kernel computes the upper triangle and mirrors it: hermitian to the bit
        assert np.array_equal(got, np.conj(got.T))


@pytest.mark.parametrize('tile', [8, 208, 708])
def test_rhs_dia_upper_tiles_form(cuda_device, coupled_kerr_4096_rhs, tile):
    """DQB_FORM_HERMITIAN_UPPER (the stage slots' layout, the form the autotuner times) at
    n = 4096: on the 32 x 32 tiles on and above the diagonal the output matches the oracle
    at 2e-6, and on and above the diagonal it equals the hermitian form's output bit for
    bit (the same arithmetic, only the lower triangle is not mirrored)."""
    w, X, ref = coupled_kerr_4096_rhs
    n = 4096
    Ls = [SparseDIA(L.offsets, L.diags[None]) for L in w['jump_ops']]
    p, keep = _problem_struct(w['H'], Ls, n, 1)
    r_d = torch.from_numpy(np.ascontiguousarray(X[None])).to('cuda')
    full = torch.empty_like(r_d)
    upper = torch.zeros_like(r_d)
    ws = torch.empty(1 << 20, dtype=torch.uint8, device='cuda')
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for form, out in ((_lib.FORM_HERMITIAN, full), (_lib.FORM_HERMITIAN_UPPER, upper)):
        _lib.check(lib.dqb_lindblad_rhs_dia_tiled(p, form, tile, r_d.data_ptr(), out.data_ptr(),
                                                  ws.data_ptr(), ws.numel(), stream), 'rhs_dia')
    got_f = full[0].cpu().numpy()
    got_u = upper[0].cpu().numpy()
    i = np.arange(n)
    tiles = i[None, :] >= 32 * (i[:, None] // 32)
    diff = np.linalg.norm((got_u - ref)[tiles]) / np.linalg.norm(ref[tiles])
    assert diff < 2e-6
    triu = i[None, :] >= i[:, None]
    assert np.array_equal(got_u[triu], got_f[triu])


def test_dia_full_size_short_solve_vs_oracle(cuda_device):
    """The n = 4096 coupled-Kerr solve (Tsit5 1e-5/1e-7) over t in [0, 0.05] against the
    oracle (complex128 state) at 1e-5 on every saved state, with equal step counts."""
    w = workloads.coupled_kerr_dia(batch=1, m=64, seed=0)
    ts = np.linspace(0.0, 0.05, 3)
    m = w['method']
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=m)
    H = (w['H'].offsets, w['H'].diags[0])
    Ls = [(L.offsets, L.diags) for L in w['jump_ops']]
    r = oracle_mesolve(H, Ls, w['rho0'], ts, rtol=m.rtol, atol=m.atol)
    assert rel_frob(res.states[0].cpu().numpy(), r.states).max() < 1e-5
    assert (int(res.infos.nsteps[0]), int(res.infos.nrejected[0])) == (r.nsteps, r.nrejected)


def test_dia_full_size_properties(cuda_device):
    """n = 4096 (two 64-level modes), one instance: trace preserved, hermitian, positive
    populations (size-independent properties; the oracle is too slow at this size)."""
    w = workloads.coupled_kerr_dia(batch=1, m=64, seed=0)
    ts = np.linspace(0.0, 0.5, 3)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=w['method'])
    st = res.states[0]
    tr = torch.diagonal(st, dim1=-2, dim2=-1).sum(-1)
    assert torch.allclose(tr.real, torch.ones_like(tr.real), atol=1e-5)
    assert float(tr.imag.abs().max()) < 1e-5
    herm = (st - st.conj().transpose(-1, -2)).abs().max().item()
    assert herm < 1e-6
    assert float(torch.diagonal(st, dim1=-2, dim2=-1).real.min()) > -1e-6
    assert int(res.infos.nrejected[0]) >= 0 and int(res.infos.nsteps[0]) > 0


def test_dia_path_dopri5_vs_oracle(cuda_device):
    """Dopri5 through the DIA stepper: two coupled Kerr modes of 10 levels (n = 100)."""
    w = workloads.coupled_kerr_dia(batch=2, m=10, seed=6)
    w['method'] = dq.Dopri5(rtol=1e-5, atol=1e-7)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], method=w['method'])
    assert int((res.infos.nsteps > 0).sum()) == 2
    for b in range(2):
        _oracle_compare(res, w, b, method='Dopri5')


@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
@pytest.mark.parametrize('hermitian', [True, False])
def test_krylov_stepper_vs_stages_and_oracle(cuda_device, method, hermitian):
    """The Krylov form of the step (an opt-in) against the stage-by-stage
    form (the reference's arithmetic, in the same FP32), on strongly driven coupled Kerr
    modes (n = 100) whose solves reject steps (a rejected step reuses its basis), with
    expectation values: step counts within two, states within the solve's tolerance of
    each other, and each form's error against a tight FP64 oracle solution (rtol and atol
    1000 times smaller) inside the tolerance: the stage form within twice the FP64
    oracle's own error, the Krylov form within max(2x the stage form's, rtol / 2).  On this
    stiff problem the Krylov form's expanded polynomial rounds ~4x worse in FP32 than the
    stages' nested evaluation (2.6e-5 against 6.0e-6 on the expectation values; a numpy
    emulation in complex64 gives the same, in complex128 the two are equal), which is why
    it is an opt-in."""
    w = workloads.coupled_kerr_dia(batch=2, m=10, seed=5, kerr=1.0, eps=3.0)
    m = (dq.Tsit5 if method == 'Tsit5' else dq.Dopri5)(rtol=1e-4, atol=1e-6)
    E = [np.diag(np.arange(100)).astype(np.complex64)]
    runs = {}
    for stepper in ('krylov', 'stages'):
        o = dq.Options(stepper=stepper, assume_hermitian=hermitian)
        runs[stepper] = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=E,
                                   method=m, options=o)
    kr, st = runs['krylov'], runs['stages']
    assert int(kr.infos.nrejected.sum()) > 0
    assert rel_frob(kr.states.cpu().numpy(), st.states.cpu().numpy()).max() < m.rtol
    dn = np.abs(kr.infos.nsteps.cpu().numpy() - st.infos.nsteps.cpu().numpy())
    assert dn.max() <= 2
    for b in range(2):
        H = (w['H'].offsets, w['H'].diags[b])
        Ls = [(L.offsets, L.diags) for L in w['jump_ops']]
        tight = oracle_mesolve(H, Ls, w['rho0'], w['tsave'], exp_ops=E, method=method,
                               rtol=m.rtol * 1e-3, atol=m.atol * 1e-3)
        err = {}
        for name, res in runs.items():
            es = rel_frob(res.states[b].cpu().numpy(), tight.states).max()
            ee = (np.abs(res.expects[b].cpu().numpy() - tight.expects)
                  / np.maximum(np.abs(tight.expects), 1.0)).max()
            err[name] = (es, ee)
        ref_s = rel_frob(oracle_mesolve(H, Ls, w['rho0'], w['tsave'], method=method, rtol=m.rtol,
                                        atol=m.atol).states, tight.states).max()
        assert err['stages'][0] <= 2 * ref_s + 1e-6, (err, ref_s)
        for i in (0, 1):
            assert err['krylov'][i] <= max(2 * err['stages'][i], 0.5 * m.rtol), err


@pytest.mark.parametrize('tile', [604, 608, 208, 0])
@pytest.mark.parametrize('m', [20, 30])
def test_rhs_dia_bulk_ragged_edges(cuda_device, m, tile):
    """The bulk-staged stencil (and the wide one) on coupled-Kerr operators whose size is not
    a multiple of the 256-column CTA band (n = 400, 900): clipped copies, zero-filled halos
    and partial row bands, against the oracle at 2e-6, with the output hermitian to the bit."""
    w = workloads.coupled_kerr_dia(batch=1, m=m, seed=3)
    n = m * m
    rng = np.random.default_rng(n)
    Y = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / (2 * n)
    X = (Y + np.conj(Y.T)).astype(np.complex64)
    Hb = (w['H'].offsets, w['H'].diags[0].astype(complex))
    Lb = [(L.offsets, L.diags.astype(complex)) for L in w['jump_ops']]
    ref = lb.vf_hermitian_dia(Hb, Lb, X.astype(complex))
    Ls = [SparseDIA(L.offsets, L.diags[None]) for L in w['jump_ops']]
    p, keep = _problem_struct(w['H'], Ls, n, 1)
    r_d = torch.from_numpy(np.ascontiguousarray(X[None])).to('cuda')
    out = torch.empty_like(r_d)
    ws = torch.empty(1 << 22, dtype=torch.uint8, device='cuda')
    lib = _lib.load()
    _lib.check(lib.dqb_lindblad_rhs_dia_tiled(p, _lib.FORM_HERMITIAN, tile, r_d.data_ptr(),
                                              out.data_ptr(), ws.data_ptr(), ws.numel(),
                                              torch.cuda.current_stream().cuda_stream), 'rhs_dia')
    got = out[0].cpu().numpy()
    assert rel_frob(got, ref) < 2e-6
    if tile >= 200:
        assert np.array_equal(got, np.conj(got.T))
