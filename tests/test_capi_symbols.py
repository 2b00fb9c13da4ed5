"""The C-ABI library builds, loads and exports every function include/*.h declares
(no compute call is made here; this runs without a GPU)."""

import ctypes
import re
from pathlib import Path

import pytest

from dynamiqs_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / 'include').glob('*.h')):
        text = re.sub(r'/\*.*?\*/', '', h.read_text(), flags=re.S)
        names += re.findall(r'^\s*(?:DQB_API\s+)?(?:const\s+)?[\w\s\*]+?\b(dqb_\w+)\s*\(', text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert 'dqb_mesolve_dense' in names and 'dqb_mesolve_dense_workspace_size' in names


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.fail(f'{_lib.LIB_PATH} not built')
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding knows every declared symbol, and nothing else
    assert set(_lib.SIGNATURES) == set(declared_functions())


def test_version_string():
    lib = _lib.load()
    assert b'sm_100a' in lib.dqb_version()


def test_argument_validation_without_gpu():
    """Entry points reject bad arguments before touching the device."""
    lib = _lib.load()
    opts = _lib.OdeOptions(method=0, form=0, rtol=1e-6, atol=1e-6, safety=0.9, factormin=0.2,
                           factormax=5.0, max_steps=10)
    outs = _lib.Outputs()
    assert lib.dqb_mesolve_dense(None, opts, outs, None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    assert lib.dqb_lindblad_rhs_dense(None, 0, None, None, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    assert lib.dqb_mesolve_dia(None, opts, outs, None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    p = _lib.DiaProblem(n=8, n_jumps=0, batch=1, h_ndiag=1)
    # h_diags missing
    assert lib.dqb_lindblad_rhs_dia(p, 0, 1, 1, None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    # operator fields suffice for a right-hand side; a too-small workspace is reported
    off = (ctypes.c_int32 * 1)(0)
    p = _lib.DiaProblem(n=8, n_jumps=0, batch=1, h_ndiag=1, h_offsets=ctypes.cast(off, ctypes.c_void_p),
                        h_diags=1)
    assert lib.dqb_lindblad_rhs_dia(p, 0, 1, 1, None, 0, None) == _lib.DQB_ERR_WORKSPACE_TOO_SMALL
    # workspace query of a complete problem is host arithmetic
    p.n_tsave, p.rho0, p.tsave = 3, 1, 1
    assert lib.dqb_mesolve_dia_workspace_size(p) > 10 * 64 * 8


def header_int_constants():
    """Every ``#define DQB_<NAME> <integer>`` of include/*.h."""
    consts = {}
    for h in sorted((ROOT / 'include').glob('*.h')):
        text = re.sub(r'/\*.*?\*/', '', h.read_text(), flags=re.S)
        for name, val in re.findall(r'^\s*#define\s+(DQB_\w+)\s+(-?\d+)\s*$', text, flags=re.M):
            consts[name] = int(val)
    return consts


def test_binding_constants_match_header():
    """The ctypes mirror's constants (named as in the header, or without its ``DQB_``
    prefix) hold the header's values: a value that drifts on one side would silently
    select another form, method, precision or stepper."""
    consts = header_int_constants()
    assert consts['DQB_FORM_HERMITIAN_UPPER'] == 2 and consts['DQB_STEPPER_KRYLOV'] == 2
    checked, wrong = 0, []
    for name, val in consts.items():
        for py in (name, name[len('DQB_'):]):
            if hasattr(_lib, py):
                checked += 1
                if getattr(_lib, py) != val:
                    wrong.append((name, val, py, getattr(_lib, py)))
                break
    assert not wrong, wrong
    for must in ('FORM_HERMITIAN', 'FORM_STANDARD', 'FORM_HERMITIAN_UPPER', 'METHOD_TSIT5',
                 'METHOD_DOPRI5', 'PREC_TF32X3', 'STEPPER_KRYLOV', 'INST_CANCELLED', 'TD_CONST'):
        assert 'DQB_' + must in consts and hasattr(_lib, must), must
    assert checked >= 20
