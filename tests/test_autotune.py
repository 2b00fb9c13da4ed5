"""Autotuner cache logic (CPU) and, on a GPU, that every tuned launch shape of the DIA
stencil gives the same right-hand side (bitwise among the register-blocked shapes, to
rounding against the generic kernel) and that the choice is cached."""

import ctypes
import json

import numpy as np
import pytest

from dynamiqs_b200 import autotune


def test_batch_bucket():
    assert [autotune.batch_bucket(b) for b in (0, 1, 2, 3, 255, 256, 5000)] == [1, 1, 2, 2, 128,
                                                                                256, 4096]


def test_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / 'tune.json'
    monkeypatch.setenv('DQB_AUTOTUNE_CACHE', str(path))
    autotune.clear_memory_cache()
    key = autotune.key_string(('dia_tile', 'gpu', 4096, 2, ((0,), ((1,),)), 8))
    with autotune._LOCK:
        autotune._MEM[key] = {'choice': 16, 'times_ms': {'4': 1.0, '8': 0.9, '16': 0.8}}
        autotune._save()
    data = json.loads(path.read_text())
    assert data[key]['choice'] == 16
    # a fresh process state reads the file back
    monkeypatch.setattr(autotune, '_LOADED', False)
    autotune._MEM.clear()
    assert autotune.lookup(key) == 16
    autotune.clear_memory_cache()


def test_disabled_returns_default(monkeypatch):
    monkeypatch.setenv('DQB_AUTOTUNE', '0')
    called = []
    got = autotune.choose(('k',), [1, 2, 3], lambda c: called.append(c), 2)
    assert got == 2 and not called


def test_dia_tune_form():
    """The DIA stencil is timed in the form the solve writes: upper tiles for the stage form
    of the hermitian form (every stepper but Krylov), whole matrices otherwise."""
    from dynamiqs_b200 import _lib
    from dynamiqs_b200.mesolve import _dia_tune_form

    H, S, U = _lib.FORM_HERMITIAN, _lib.FORM_STANDARD, _lib.FORM_HERMITIAN_UPPER
    assert _dia_tune_form(H, _lib.STEPPER_AUTO) == U
    assert _dia_tune_form(H, _lib.STEPPER_STAGES) == U
    assert _dia_tune_form(H, _lib.STEPPER_KRYLOV) == H
    for st in (_lib.STEPPER_AUTO, _lib.STEPPER_STAGES, _lib.STEPPER_KRYLOV):
        assert _dia_tune_form(S, st) == S


@pytest.mark.gpu
def test_dia_tiles_equal_and_cached(cuda_device, tmp_path, monkeypatch):
    import torch

    from dynamiqs_b200 import _lib, workloads
    from dynamiqs_b200.mesolve import DIA_STENCIL_SHAPES, MESolveB200Integrator, make_batch_plan

    monkeypatch.setenv('DQB_AUTOTUNE_CACHE', str(tmp_path / 'tune.json'))
    autotune.clear_memory_cache()
    w = workloads.coupled_kerr_dia(batch=2, m=24, seed=1)
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                  options=__import__('dynamiqs_b200').Options(), H=w['H'],
                                  Ls=w['jump_ops'], Es=None, plan=plan)
    prep = integ.prepare()
    assert integ._tuned['tile'] in DIA_STENCIL_SHAPES
    assert (tmp_path / 'tune.json').exists()
    lib = _lib.load()
    n = w['H'].diags.shape[-1]
    rng = np.random.default_rng(0)
    Y = rng.normal(size=(2, n, n)) + 1j * rng.normal(size=(2, n, n))
    rho = torch.from_numpy((Y @ np.conj(np.swapaxes(Y, -1, -2)) / n).astype(np.complex64)).cuda()
    outs = []
    for tile in DIA_STENCIL_SHAPES:
        out = torch.empty_like(rho)
        _lib.check(lib.dqb_lindblad_rhs_dia_tiled(
            ctypes.byref(prep.prob), _lib.FORM_HERMITIAN, tile, rho.data_ptr(), out.data_ptr(),
            prep.bufs['workspace'].data_ptr(), prep.ws_bytes,
            torch.cuda.current_stream().cuda_stream), 'rhs_dia_tiled')
        outs.append(out.cpu().numpy())
    # the generic, tiled and staged kernels sum the same terms in different orders: equal
    # to rounding; the tiled shapes among themselves: bitwise
    assert np.array_equal(outs[1], outs[2]) and np.array_equal(outs[2], outs[3])
    for o in outs[1:]:  # the right-hand-side bar of the parity tests: 2e-6 relative Frobenius
        assert np.linalg.norm(outs[0] - o) <= 2e-6 * np.linalg.norm(o)
    autotune.clear_memory_cache()
