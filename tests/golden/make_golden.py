"""Extract the known answers for the mesolve hot path from the reference's own docs.

Run from the repository root with the path of a read-only checkout of the reference
as the only argument::

    python tests/golden/make_golden.py <reference checkout>

It reads printed outputs (step counts, final states, expectation values) from the
reference's README, docstrings and docs pages, and writes ``known_answers.json`` next to
this script with the source file:line of every value.  The systems these outputs belong
to are described in the JSON (operators, tolerances, save times) so the tests can
re-run them through the oracle and the GPU path.
"""

from __future__ import annotations

import json
import re
import sys
from pathlib import Path


def _find(path: Path, pattern: str):
    lines = path.read_text().splitlines()
    rx = re.compile(pattern)
    for i, line in enumerate(lines, start=1):
        m = rx.search(line)
        if m:
            return m, i
    raise RuntimeError(f'pattern {pattern!r} not found in {path}')


def main(ref: str) -> None:
    ref = Path(ref)
    out = {}
    steps_rx = r'Infos\s*:\s*(\d+) steps \((\d+) accepted, (\d+) rejected\)'

    m, ln = _find(ref / 'README.md', steps_rx)
    out['readme_lossy_oscillator'] = {
        'source': f'README.md:{ln}',
        'system': {'n': 16, 'H': 'omega * a^+ a', 'omega': 1.0, 'jump_ops': ['sqrt(kappa) a'],
                   'kappa': 0.1, 'rho0': 'coherent(n, alpha0)', 'alpha0': 1.0,
                   'tsave': 'linspace(0, 2 pi, 101)', 'method': 'Tsit5', 'rtol': 1e-6,
                   'atol': 1e-6},
        'nsteps': int(m[1]), 'naccepted': int(m[2]), 'nrejected': int(m[3]),
    }

    m, ln = _find(ref / 'dynamiqs/integrators/apis/mesolve.py', steps_rx)
    out['mesolve_docstring'] = {
        'source': f'dynamiqs/integrators/apis/mesolve.py:{ln}',
        'system': {'n': 16, 'H': 'a^+ a', 'jump_ops': ['a'], 'rho0': 'coherent(n, 1.0)',
                   'tsave': 'linspace(0, 1, 11)', 'method': 'Tsit5', 'rtol': 1e-6,
                   'atol': 1e-6},
        'nsteps': int(m[1]), 'naccepted': int(m[2]), 'nrejected': int(m[3]),
    }

    m, ln = _find(ref / 'docs/documentation/basics/workflow.md', steps_rx)
    out['workflow_dopri5_sesolve'] = {
        'source': f'docs/documentation/basics/workflow.md:{ln}',
        'system': {'n': 2, 'H': 'delta sigmaz + Omega sigmax', 'delta': 0.3, 'Omega': 1.0,
                   'psi0': 'fock(2, 0)', 'tsave': 'linspace(0, 10, 101)',
                   'method': 'Dopri5', 'rtol': 1e-6, 'atol': 1e-8,
                   'equation': 'Schroedinger (same RK engine)'},
        'nsteps': int(m[1]), 'naccepted': int(m[2]), 'nrejected': int(m[3]),
    }

    m, ln = _find(ref / 'dynamiqs/integrators/apis/sesolve.py', steps_rx)
    out['sesolve_docstring'] = {
        'source': f'dynamiqs/integrators/apis/sesolve.py:{ln}',
        'system': {'n': 16, 'H': 'a^+ a', 'psi0': 'coherent(n, 1.0)',
                   'tsave': 'linspace(0, 1, 11)', 'method': 'Tsit5', 'rtol': 1e-6,
                   'atol': 1e-6, 'equation': 'Schroedinger'},
        'nsteps': int(m[1]), 'naccepted': int(m[2]), 'nrejected': int(m[3]),
    }

    p = ref / 'docs/documentation/basics/open-systems.md'
    m0, ln0 = _find(p, r'^\s*\[\[([-\d.]+)\+0\.j\s+0\.\s*\+0\.j\]')
    m1, _ = _find(p, r'^\s*\[\s*0\.\s*\+0\.j\s+([-\d.]+)\+0\.j\]\]')
    out['open_systems_qubit_decay'] = {
        'source': f'docs/documentation/basics/open-systems.md:{ln0}',
        'system': {'n': 2, 'H': 'sigmaz', 'jump_ops': ['sigmam'], 'rho0': 'excited()',
                   'tsave': 'linspace(0, 1, 11)', 'method': 'Tsit5', 'rtol': 1e-6,
                   'atol': 1e-6},
        'final_diag': [float(m0[1]), float(m1[1])], 'decimals': 3,
    }

    m, ln = _find(ref / 'docs/documentation/advanced_examples/kerr-oscillator.md',
                  r'Array\(([-\d.]+)\+0\.j')
    out['kerr_oscillator_photon_number'] = {
        'source': f'docs/documentation/advanced_examples/kerr-oscillator.md:{ln}',
        'system': {'n': 32, 'H': '-K a^+ a^+ a a + epsilon (a + a^+)', 'K': 1.0,
                   'epsilon': 3.0, 'jump_ops': ['sqrt(kappa) a'], 'kappa': 1.5,
                   'rho0': 'coherent(n, alpha0)', 'alpha0': 2.0,
                   'tsave': 'linspace(0, 5, 201)', 'method': 'Tsit5', 'rtol': 1e-6,
                   'atol': 1e-6},
        'final_number': float(m[1]), 'decimals': 3,
    }

    out['ocavity_test_system'] = {
        'source': 'tests/systems/open_system.py:172-182,233-240',
        'system': {'n': 8, 'H': 'delta a^+ a', 'delta': '2 pi', 'jump_ops': ['sqrt(kappa) a'],
                   'kappa': '2 pi', 'rho0': 'coherent(n, alpha0)', 'alpha0': 0.5,
                   'tsave': 'linspace(0, 0.3, 11)', 'exp_ops': ['position', 'momentum']},
        'analytic': 'rho(t) = |alpha(t)><alpha(t)|, alpha(t) = alpha0 exp(-i delta t - kappa t / 2)',
        'tolerances': {'ysave_atol': 1e-3, 'esave_rtol': 1e-3, 'esave_atol': 1e-4,
                       'source': 'tests/integrator_tester.py:17-47'},
    }

    dest = Path(__file__).with_name('known_answers.json')
    dest.write_text(json.dumps(out, indent=2) + '\n')
    print(f'wrote {dest}')


if __name__ == '__main__':
    if len(sys.argv) != 2:
        sys.exit('usage: python tests/golden/make_golden.py <reference checkout>')
    main(sys.argv[1])
