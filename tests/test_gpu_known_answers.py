"""The device controllers reproduce the step counts the reference prints for its own
examples, exactly, on every solve path:

* README lossy oscillator (README.md:48-76): "40 steps (40 accepted, 0 rejected)";
* ``mesolve`` docstring (dynamiqs/integrators/apis/mesolve.py:204-227): "9 steps
  (9 accepted, 0 rejected)".

The shared-memory kernel (n <= 64) runs them through the public ``mesolve``; the GEMM
path's stepper and the DIA stepper run the same problems through their own entry
points (``dqb_mesolve_dense_large``, ``dqb_mesolve_dia``), whose controller code is
separate."""

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib
from dynamiqs_b200 import operators as ops
from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan
from tests.systems import GOLDEN

pytestmark = pytest.mark.gpu


def _readme(layout):
    n = 16
    a = ops.destroy(n, layout=layout)
    return (ops.dag(a) @ a, [a * np.float32(np.sqrt(0.1))], ops.coherent(n, 1.0),
            np.linspace(0, 2 * np.pi, 101))


def _docstring(layout):
    n = 16
    a = ops.destroy(n, layout=layout)
    return ops.dag(a) @ a, [a], ops.coherent(n, 1.0), np.linspace(0, 1.0, 11)


CASES = {'readme_lossy_oscillator': _readme, 'mesolve_docstring': _docstring}


def _counts(res):
    i = res.infos
    return int(i.nsteps), int(i.naccepted), int(i.nrejected)


def _golden(key):
    g = GOLDEN[key]
    return g['nsteps'], g['naccepted'], g['nrejected']


@pytest.mark.parametrize('layout', ['dense', 'dia'])
@pytest.mark.parametrize('key', list(CASES))
def test_public_mesolve_counts(cuda_device, key, layout):
    H, Ls, psi0, ts = CASES[key](layout)
    res = dq.mesolve(H, Ls, psi0, ts)  # default Tsit5(rtol=1e-6, atol=1e-6)
    assert _counts(res) == _golden(key)


@pytest.mark.parametrize('path', ['dense_large', 'dia'])
@pytest.mark.parametrize('key', list(CASES))
def test_stepper_counts(cuda_device, key, path):
    H, Ls, psi0, ts = CASES[key]('dia' if path == 'dia' else 'dense')
    plan = make_batch_plan(H, Ls, psi0, True)
    integ = MESolveB200Integrator(ts=ts, y0=psi0, method=dq.Tsit5(), gradient=None,
                                  options=dq.Options(), H=H, Ls=Ls, Es=[], plan=plan)
    lib = _lib.load()
    res = integ._run_dense_large(lib) if path == 'dense_large' else integ._run_dia(lib)
    assert _counts(res) == _golden(key)
