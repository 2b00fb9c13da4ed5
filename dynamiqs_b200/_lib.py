"""ctypes binding of ``libdqb200.so`` (the C ABI declared in ``include/dqb200.h``).

The shared library is built in-tree (``dynamiqs_b200/csrc/Makefile``) and loaded from
this package directory.  There is no fallback: if the library is missing, or was built
without CUDA support, every solve raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / 'libdqb200.so'

# return codes
DQB_OK = 0
DQB_ERR_INVALID_ARGUMENT = 1
DQB_ERR_UNSUPPORTED = 2
DQB_ERR_WORKSPACE_TOO_SMALL = 3
DQB_ERR_CUDA = 4
DQB_ERR_SCRATCH_TOO_SMALL = 5
_RC_NAMES = {
    DQB_ERR_INVALID_ARGUMENT: 'invalid argument',
    DQB_ERR_UNSUPPORTED: 'unsupported problem size or option',
    DQB_ERR_WORKSPACE_TOO_SMALL: 'workspace too small',
    DQB_ERR_CUDA: 'CUDA launch error',
    DQB_ERR_SCRATCH_TOO_SMALL: 'problem needs more than the static scratch array',
}

# per-instance status
INST_OK = 0
INST_MAX_STEPS = 1
INST_NONFINITE = 2
INST_NOT_HERMITIAN = 3
INST_CANCELLED = 4

METHOD_TSIT5 = 0
METHOD_DOPRI5 = 1
FORM_HERMITIAN = 0
FORM_STANDARD = 1
FORM_HERMITIAN_UPPER = 2  # DIA right-hand-side entry points only: upper 32 x 32 tiles
PREC_FP32 = 0
PREC_TF32X3 = 1
PREC_BF16X3 = 2
PREC_TF32 = 3
PREC_F16X3 = 4
STEPPER_AUTO = 0
STEPPER_STAGES = 1
STEPPER_KRYLOV = 2
STEPPERS = {'auto': STEPPER_AUTO, 'stages': STEPPER_STAGES, 'krylov': STEPPER_KRYLOV}
PRECISIONS = {'fp32': PREC_FP32, 'tf32x3': PREC_TF32X3, 'bf16x3': PREC_BF16X3, 'tf32': PREC_TF32,
              'f16x3': PREC_F16X3}


class OdeOptions(ctypes.Structure):
    _fields_ = [
        ('method', ctypes.c_int32),
        ('form', ctypes.c_int32),
        ('rtol', ctypes.c_double),
        ('atol', ctypes.c_double),
        ('safety', ctypes.c_double),
        ('factormin', ctypes.c_double),
        ('factormax', ctypes.c_double),
        ('max_steps', ctypes.c_int64),
        ('t0', ctypes.c_double),
        ('save_states', ctypes.c_int32),
        ('check_hermitian', ctypes.c_int32),
        ('precision', ctypes.c_int32),
        ('tile', ctypes.c_int32),
        ('stepper', ctypes.c_int32),
    ]


class Outputs(ctypes.Structure):
    _fields_ = [
        ('states', ctypes.c_void_p),
        ('expects', ctypes.c_void_p),
        ('infos', ctypes.c_void_p),
        ('status', ctypes.c_void_p),
    ]


class DenseProblem(ctypes.Structure):
    _fields_ = [
        ('n', ctypes.c_int32),
        ('n_jumps', ctypes.c_int32),
        ('n_exp', ctypes.c_int32),
        ('n_tsave', ctypes.c_int32),
        ('batch', ctypes.c_int64),
        ('H', ctypes.c_void_p),
        ('L', ctypes.c_void_p),
        ('rho0', ctypes.c_void_p),
        ('rho0_is_ket', ctypes.c_int32),
        ('E', ctypes.c_void_p),
        ('tsave', ctypes.c_void_p),
        ('H_index', ctypes.c_void_p),
        ('L_index', ctypes.c_void_p),
        ('rho0_index', ctypes.c_void_p),
        ('start_order', ctypes.c_void_p),
    ]


class DiaProblem(ctypes.Structure):
    _fields_ = [
        ('n', ctypes.c_int32),
        ('n_jumps', ctypes.c_int32),
        ('n_exp', ctypes.c_int32),
        ('n_tsave', ctypes.c_int32),
        ('batch', ctypes.c_int64),
        ('h_ndiag', ctypes.c_int32),
        ('h_offsets', ctypes.c_void_p),
        ('h_diags', ctypes.c_void_p),
        ('l_ndiag', ctypes.c_void_p),
        ('l_offsets', ctypes.c_void_p),
        ('l_diags', ctypes.c_void_p),
        ('rho0', ctypes.c_void_p),
        ('rho0_is_ket', ctypes.c_int32),
        ('E', ctypes.c_void_p),
        ('tsave', ctypes.c_void_p),
        ('H_index', ctypes.c_void_p),
        ('L_index', ctypes.c_void_p),
        ('rho0_index', ctypes.c_void_p),
    ]


class RaggedInstance(ctypes.Structure):
    _fields_ = [
        ('n', ctypes.c_int32),
        ('n_jumps', ctypes.c_int32),
        ('n_exp', ctypes.c_int32),
        ('n_tsave', ctypes.c_int32),
        ('rho0_is_ket', ctypes.c_int32),
        ('save_states', ctypes.c_int32),
        ('t0', ctypes.c_double),
        ('H', ctypes.c_void_p),
        ('L', ctypes.c_void_p),
        ('rho0', ctypes.c_void_p),
        ('E', ctypes.c_void_p),
        ('tsave', ctypes.c_void_p),
        ('states', ctypes.c_void_p),
        ('expects', ctypes.c_void_p),
        ('infos', ctypes.c_void_p),
        ('status', ctypes.c_void_p),
        ('cancel', ctypes.c_void_p),
    ]


TD_PWC = 0
TD_WAVE = 1
TD_CONST = 2
TD_MAX_TERMS = 4
DIA_MAX_HNH_DIAGS = 64  # DQB_DIA_MAX_HNH_DIAGS


class TdTerm(ctypes.Structure):
    _fields_ = [
        ('kind', ctypes.c_int32),
        ('n_times', ctypes.c_int32),
        ('times', ctypes.c_void_p),
        ('values', ctypes.c_void_p),
        ('value_index', ctypes.c_void_p),
        ('amp_re', ctypes.c_double),
        ('amp_im', ctypes.c_double),
        ('omega', ctypes.c_double),
        ('phase', ctypes.c_double),
        ('t_center', ctypes.c_double),
        ('sigma', ctypes.c_double),
        ('t_start', ctypes.c_double),
        ('t_end', ctypes.c_double),
    ]


class TdHamiltonian(ctypes.Structure):
    _fields_ = [
        ('n_terms', ctypes.c_int32),
        ('ops', ctypes.c_void_p),
        ('terms', ctypes.POINTER(TdTerm)),
        ('n_jump_ts', ctypes.c_int32),
        ('jump_ts', ctypes.c_void_p),
        ('jump_terms', ctypes.POINTER(TdTerm)),
    ]


class Tape(ctypes.Structure):
    _fields_ = [('t', ctypes.c_void_p), ('h', ctypes.c_void_p), ('y', ctypes.c_void_p),
                ('capacity', ctypes.c_int32)]


class Cotangents(ctypes.Structure):
    _fields_ = [('states', ctypes.c_void_p), ('expects', ctypes.c_void_p)]


class Gradients(ctypes.Structure):
    _fields_ = [('rho0', ctypes.c_void_p), ('H', ctypes.c_void_p), ('L', ctypes.c_void_p)]


# Every symbol include/dqb200.h declares, with (restype, argtypes).
_P = ctypes.c_void_p
SIGNATURES = {
    'dqb_mesolve_dense_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64]),
    'dqb_mesolve_dense': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                         ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_mesolve_dense_td': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(TdHamiltonian),
                                            ctypes.POINTER(OdeOptions), ctypes.POINTER(Outputs), _P,
                                            ctypes.c_size_t, _P]),
    'dqb_mesolve_dense_noalloc': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                                 ctypes.POINTER(Outputs), _P]),
    'dqb_lindblad_rhs_dense': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.c_int32, _P, _P, _P]),
    'dqb_lindblad_rhs_dense_prec': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.c_int32,
                                                   ctypes.c_int32, _P, _P, _P, ctypes.c_size_t, _P]),
    'dqb_mesolve_dense_large_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32,
                                                                 ctypes.c_int32, ctypes.c_int32,
                                                                 ctypes.c_int64]),
    'dqb_mesolve_dense_large': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                               ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_lindblad_rhs_dense_large': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.c_int32, _P,
                                                    _P, _P, ctypes.c_size_t, _P]),
    'dqb_lindblad_rhs_dense_large_prec': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.c_int32,
                                                         ctypes.c_int32, _P, _P, _P, ctypes.c_size_t, _P]),
    'dqb_mesolve_ragged_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64]),
    'dqb_mesolve_ragged': (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.POINTER(OdeOptions), _P, ctypes.c_size_t, _P]),
    'dqb_mesolve_dense_large_ragged_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32,
                                                                        ctypes.c_int32, ctypes.c_int32,
                                                                        ctypes.c_int64]),
    'dqb_mesolve_dense_large_ragged': (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_int32,
                                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                      ctypes.POINTER(OdeOptions), _P, ctypes.c_size_t, _P]),
    'dqb_mesolve_dia_workspace_size': (ctypes.c_size_t, [ctypes.POINTER(DiaProblem)]),
    'dqb_mesolve_dense_large_td_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32,
                                                                    ctypes.c_int32, ctypes.c_int32,
                                                                    ctypes.c_int64]),
    'dqb_mesolve_dense_large_td': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(TdHamiltonian),
                                                  ctypes.POINTER(OdeOptions), ctypes.POINTER(Outputs), _P,
                                                  ctypes.c_size_t, _P]),
    'dqb_mesolve_dia_td': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.POINTER(TdHamiltonian),
                                          ctypes.POINTER(OdeOptions), ctypes.POINTER(Outputs), _P,
                                          ctypes.c_size_t, _P]),
    'dqb_mesolve_dia': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.POINTER(OdeOptions),
                                       ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_lindblad_rhs_dia': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.c_int32, _P, _P, _P,
                                            ctypes.c_size_t, _P]),
    'dqb_lindblad_rhs_dia_tiled': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.c_int32,
                                                  ctypes.c_int32, _P, _P, _P, ctypes.c_size_t, _P]),
    'dqb_dense_small_max_n': (ctypes.c_int32, [ctypes.c_int32]),
    'dqb_set_tc_wait_limit_ns': (None, [ctypes.c_uint64]),
    'dqb_mesolve_dense_tape_bytes': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64]),
    'dqb_mesolve_dense_taped': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                               ctypes.POINTER(Outputs), ctypes.POINTER(Tape), _P,
                                               ctypes.c_size_t, _P]),
    'dqb_mesolve_dense_adjoint_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32,
                                                                   ctypes.c_int64]),
    'dqb_mesolve_dense_adjoint': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                                 ctypes.POINTER(Tape), _P, ctypes.POINTER(Cotangents),
                                                 ctypes.POINTER(Gradients), _P, ctypes.c_size_t, _P]),
    'dqb_probe_bounded_wait': (ctypes.c_int, [ctypes.c_uint64, _P, _P]),
    'dqb_sesolve_dense_workspace_size': (ctypes.c_size_t, []),
    'dqb_sesolve_dense': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                         ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_schrodinger_rhs_dense': (ctypes.c_int, [ctypes.POINTER(DenseProblem), _P, _P, _P]),
    'dqb_sesolve_large_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32,
                                                           ctypes.c_int32, ctypes.c_int64]),
    'dqb_sesolve_dense_large': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(OdeOptions),
                                               ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_sesolve_dia': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.POINTER(OdeOptions),
                                       ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_sesolve_large_td_workspace_size': (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                                              ctypes.c_int32, ctypes.c_int64]),
    'dqb_sesolve_dense_large_td': (ctypes.c_int, [ctypes.POINTER(DenseProblem), ctypes.POINTER(TdHamiltonian),
                                                  ctypes.POINTER(OdeOptions), ctypes.POINTER(Outputs), _P,
                                                  ctypes.c_size_t, _P]),
    'dqb_sesolve_dia_td': (ctypes.c_int, [ctypes.POINTER(DiaProblem), ctypes.POINTER(TdHamiltonian),
                                          ctypes.POINTER(OdeOptions), ctypes.POINTER(Outputs), _P,
                                          ctypes.c_size_t, _P]),
    'dqb_mesolve_vectorized': (ctypes.c_int, [ctypes.POINTER(DenseProblem), _P, ctypes.POINTER(OdeOptions),
                                              ctypes.POINTER(Outputs), _P, ctypes.c_size_t, _P]),
    'dqb_version': (ctypes.c_char_p, []),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f'{LIB_PATH} is missing: build it with `make -C dynamiqs_b200/csrc` '
            '(or `python -c "import __graft_entry__ as g; g.build()"`). '
            'dynamiqs_b200 has no CPU fallback.')
    lib = ctypes.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != DQB_OK:
        raise RuntimeError(f'{what} failed: {_RC_NAMES.get(rc, rc)} (code {rc})')
