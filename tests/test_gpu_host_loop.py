"""The RK loop of the large-problem paths (dense GEMM path, n > 64, and sparse DIA) runs
as a CUDA-graph WHILE node by default and, with DQB_HOST_LOOP=1, from the host (the form
profilers can see).  Both run the same kernels in the same order, so their results are
bitwise equal; the host-driven run happens in a child process because the switch is read
once per process."""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
import dynamiqs_b200 as dq
from dynamiqs_b200 import workloads
out = {{}}
w = workloads.transmon_cavity(batch=2, nq=2, nc=40, seed=5)
w['tsave'] = np.linspace(0.0, 1.0, 5)
r = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'], method=w['method'])
out['dense'] = [r.states.cpu().numpy().view(np.float32).tolist(), r.infos.nsteps.cpu().tolist()]
w = workloads.coupled_kerr_dia(batch=1, m=10, seed=2)
w['tsave'] = np.linspace(0.0, 0.5, 3)
r = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], method=w['method'])
out['dia'] = [r.states.cpu().numpy().view(np.float32).tolist(), r.infos.nsteps.cpu().tolist()]
print('RESULT' + json.dumps(out))
'''


def _solve_here():
    out = {}
    w = workloads.transmon_cavity(batch=2, nq=2, nc=40, seed=5)
    w['tsave'] = np.linspace(0.0, 1.0, 5)
    r = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                   method=w['method'])
    out['dense'] = (r.states.cpu().numpy(), r.infos.nsteps.cpu().numpy())
    w = workloads.coupled_kerr_dia(batch=1, m=10, seed=2)
    w['tsave'] = np.linspace(0.0, 0.5, 3)
    r = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], method=w['method'])
    out['dia'] = (r.states.cpu().numpy(), r.infos.nsteps.cpu().numpy())
    return out


def test_host_driven_loop_equals_graph_loop(cuda_device):
    import gc

    import torch

    here = _solve_here()
    # the child needs device memory that earlier tests of this process may still hold in
    # torch's cache (a serving arena takes most of the device)
    gc.collect()
    torch.cuda.empty_cache()
    env = dict(os.environ, DQB_HOST_LOOP='1')
    proc = subprocess.run([sys.executable, '-c', _CHILD.format(root=ROOT)], env=env,
                          capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    line = [x for x in proc.stdout.splitlines() if x.startswith('RESULT')][-1]
    child = json.loads(line[len('RESULT'):])
    for key in ('dense', 'dia'):
        states, nsteps = here[key]
        c_states = np.asarray(child[key][0], dtype=np.float32).view(np.complex64)
        assert c_states.shape == states.shape
        assert np.array_equal(c_states, states), key
        assert np.array_equal(np.asarray(child[key][1]), nsteps), key
