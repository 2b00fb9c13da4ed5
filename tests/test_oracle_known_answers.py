"""Pin the oracle against the reference's own known answers (tests/golden/
known_answers.json, extracted from its docs by tests/golden/make_golden.py) and the
analytic solutions its test-suite uses."""

import numpy as np
import pytest

from dynamiqs_b200 import operators as ops
from oracle.mesolve import mesolve, sesolve
from tests.systems import GOLDEN, coherent_alpha_t, docstring_oscillator, ocavity, readme_oscillator


def _run(p, **kw):
    return mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'], rtol=p['rtol'],
                   atol=p['atol'], **kw)


@pytest.mark.parametrize('time_dtype', [np.float64, np.float32])
@pytest.mark.parametrize('dtype', [np.complex128, np.complex64])
def test_readme_oscillator(dtype, time_dtype):
    g = GOLDEN['readme_lossy_oscillator']
    r = _run(readme_oscillator(), dtype=dtype, time_dtype=time_dtype)
    assert (r.nsteps, r.naccepted, r.nrejected) == (g['nsteps'], g['naccepted'],
                                                    g['nrejected'])
    t = np.linspace(0, 2 * np.pi, 101)
    true = np.stack([ops.coherent_dm(16, coherent_alpha_t(1.0, 1.0, 0.1, s)) for s in t])
    err = np.linalg.norm(r.states - true, axis=(-2, -1))
    assert err.max() < 1e-4


def test_docstring_oscillator():
    g = GOLDEN['mesolve_docstring']
    r = _run(docstring_oscillator())
    assert (r.nsteps, r.naccepted, r.nrejected) == (g['nsteps'], g['naccepted'],
                                                    g['nrejected'])
    true = ops.coherent_dm(16, coherent_alpha_t(1.0, 1.0, 1.0, 1.0))
    assert np.linalg.norm(r.states[-1] - true) < 1e-4


def test_workflow_dopri5_rejections():
    g = GOLDEN['workflow_dopri5_sesolve']
    sx = np.array([[0, 1], [1, 0]], complex)
    sz = np.array([[1, 0], [0, -1]], complex)
    out = sesolve(0.3 * sz + 1.0 * sx, np.array([[1], [0]], complex), np.linspace(0, 10, 101),
                  method='Dopri5', rtol=1e-6, atol=1e-8)
    assert (out.nsteps, out.naccepted, out.nrejected) == (g['nsteps'], g['naccepted'],
                                                          g['nrejected'])


def test_qubit_decay_final_state():
    g = GOLDEN['open_systems_qubit_decay']
    sz = np.array([[1, 0], [0, -1]], np.complex64)
    sm = np.array([[0, 0], [1, 0]], np.complex64)
    r = mesolve(sz, [sm], np.array([[1], [0]], np.complex64), np.linspace(0, 1, 11))
    np.testing.assert_allclose(np.round(np.diag(r.states[-1]).real, g['decimals']),
                               g['final_diag'])


def test_kerr_photon_number():
    g = GOLDEN['kerr_oscillator_photon_number']
    n = 32
    a = ops.destroy(n, layout='dense')
    ad = ops.dag(a)
    H = -1.0 * (ad @ ad @ a @ a) + 3.0 * (a + ad)
    r = mesolve(H, [np.sqrt(1.5) * a], ops.coherent(n, 2.0), np.linspace(0, 5, 201))
    nbar = ops.expect(ad @ a, r.states[-1]).real
    assert round(float(nbar), g['decimals']) == g['final_number']


@pytest.mark.parametrize('layout', ['dense', 'dia'])
@pytest.mark.parametrize('form', ['hermitian', 'standard', 'vectorized'])
def test_ocavity_analytic(layout, form):
    """``TestMESolveAdaptive.test_correctness`` (reference tests/mesolve/
    test_adaptive.py:13-23) with its tolerances (tests/integrator_tester.py:17-47)."""
    p = ocavity(layout)
    if form != 'hermitian' and layout == 'dia':
        pass  # DIA operators are densified by the oracle for these forms
    H = (p['H'].offsets, p['H'].diags) if layout == 'dia' else p['H']
    Ls = [(L.offsets, L.diags) if layout == 'dia' else L for L in p['jump_ops']]
    Es = [E.to_dense() if layout == 'dia' else E for E in p['exp_ops']]
    r = mesolve(H, Ls, p['rho0'], p['tsave'], exp_ops=Es, form=form)
    errs = np.linalg.norm(r.states - p['true_states'], axis=(-2, -1))
    assert np.all(errs <= 1e-3)
    np.testing.assert_allclose(r.expects, p['true_expects'], rtol=1e-3, atol=1e-4)


@pytest.mark.parametrize('dtype', [np.complex128, np.complex64])
def test_sesolve_docstring(dtype):
    """``dq.sesolve`` docstring (dynamiqs/integrators/apis/sesolve.py): 11 steps, none
    rejected -- a fourth printed count, reproduced by the controller pinned on the other
    three."""
    g = GOLDEN['sesolve_docstring']
    a = ops.destroy(16, layout='dense')
    out = sesolve(ops.dag(a) @ a, ops.coherent(16, 1.0), np.linspace(0, 1.0, 11), dtype=dtype)
    assert (out.nsteps, out.naccepted, out.nrejected) == (g['nsteps'], g['naccepted'],
                                                          g['nrejected'])
