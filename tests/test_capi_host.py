"""Host-only behaviour of the C ABI (no GPU, nothing launched): workspace-size arithmetic and
the argument checks every entry point makes before it touches the device -- invalid
arguments come back as DQB_* status codes, never as a crash."""

import ctypes

import numpy as np

from dynamiqs_b200 import _lib


def _dense(**kw):
    p = _lib.DenseProblem(n=8, n_jumps=1, n_exp=0, n_tsave=2, batch=1, H=1, L=1, rho0=1, tsave=1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _opts(**kw):
    o = _lib.OdeOptions(method=_lib.METHOD_TSIT5, form=_lib.FORM_HERMITIAN, rtol=1e-6, atol=1e-6,
                        safety=0.9, factormin=0.2, factormax=5.0, max_steps=1000, save_states=1)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def test_large_workspace_size_arithmetic():
    lib = _lib.load()
    n, K, nE, nt, B = 130, 2, 1, 5, 3
    got = lib.dqb_mesolve_dense_large_workspace_size(n, K, nE, nt, B)
    nn = n * n * 8
    # 10 RK slots, Hnh, K product buffers and one sum buffer per instance, plus the
    # controller records and FP64 expectation accumulators (256-byte aligned blocks)
    assert got >= B * (10 + 1 + K + 1) * nn
    assert got < B * (10 + 1 + K + 1) * nn + 64 * 1024
    assert lib.dqb_mesolve_dense_large_workspace_size(1, K, nE, nt, B) == 0  # n < 2
    assert lib.dqb_mesolve_dense_large_workspace_size(n, K, nE, 0, B) == 0   # no tsave
    assert lib.dqb_mesolve_dense_large_ragged_workspace_size(n, K, nE, nt, B) == got


def test_dia_workspace_size_and_limits():
    lib = _lib.load()
    n = 100
    h_off = (ctypes.c_int32 * 3)(-1, 0, 1)
    l_nd = (ctypes.c_int32 * 1)(1)
    l_off = (ctypes.c_int32 * 1)(1)
    vp = ctypes.c_void_p
    p = _lib.DiaProblem(n=n, n_jumps=1, n_exp=0, n_tsave=3, batch=2, h_ndiag=3,
                        h_offsets=ctypes.cast(h_off, vp), h_diags=1, l_ndiag=ctypes.cast(l_nd, vp),
                        l_offsets=ctypes.cast(l_off, vp), l_diags=1, rho0=1, tsave=1)
    ws = lib.dqb_mesolve_dia_workspace_size(p)
    assert ws >= 2 * 10 * n * n * 8  # ten n x n slots per instance
    bad = (ctypes.c_int32 * 3)(-n, 0, 1)  # an offset outside (-n, n)
    p.h_offsets = ctypes.cast(bad, vp)
    assert lib.dqb_mesolve_dia_workspace_size(p) == 0


def test_solves_reject_invalid_arguments_before_any_launch():
    lib = _lib.load()
    outs = _lib.Outputs(states=1, expects=0, infos=1, status=1)
    cases = [
        (None, _opts()),
        (_dense(), None),
        (_dense(n=0), _opts()),
        (_dense(n_tsave=0), _opts()),
        (_dense(batch=-1), _opts()),
        (_dense(H=0), _opts()),
        (_dense(n_exp=1, E=0), _opts()),
        (_dense(), _opts(method=7)),
        (_dense(), _opts(form=5)),
        (_dense(), _opts(rtol=-1.0)),
        (_dense(), _opts(max_steps=-1)),
    ]
    for p, o in cases:
        pp = ctypes.byref(p) if p is not None else None
        po = ctypes.byref(o) if o is not None else None
        assert lib.dqb_mesolve_dense(pp, po, ctypes.byref(outs), None, 0, None) == \
            _lib.DQB_ERR_INVALID_ARGUMENT
        assert lib.dqb_mesolve_dense_noalloc(pp, po, ctypes.byref(outs), None) == \
            _lib.DQB_ERR_INVALID_ARGUMENT
    # missing outputs
    empty = _lib.Outputs(states=0, expects=0, infos=0, status=0)
    assert lib.dqb_mesolve_dense(ctypes.byref(_dense()), ctypes.byref(_opts()), ctypes.byref(empty),
                                 None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    assert lib.dqb_mesolve_dense_large(ctypes.byref(_dense(n=100)), ctypes.byref(_opts()),
                                       ctypes.byref(empty), None, 0, None) == \
        _lib.DQB_ERR_INVALID_ARGUMENT


def test_large_path_rejects_bad_precision_and_small_workspace():
    lib = _lib.load()
    outs = _lib.Outputs(states=1, expects=0, infos=1, status=1)
    p = _dense(n=100)
    assert lib.dqb_mesolve_dense_large(ctypes.byref(p), ctypes.byref(_opts(precision=9)),
                                       ctypes.byref(outs), None, 0, None) == \
        _lib.DQB_ERR_INVALID_ARGUMENT
    # tensor-core products need the hermitian form and an even n
    assert lib.dqb_mesolve_dense_large(ctypes.byref(_dense(n=101)),
                                       ctypes.byref(_opts(precision=_lib.PREC_TF32X3)),
                                       ctypes.byref(outs), None, 0, None) == _lib.DQB_ERR_UNSUPPORTED
    assert lib.dqb_mesolve_dense_large(ctypes.byref(p), ctypes.byref(_opts(form=_lib.FORM_STANDARD,
                                                                             precision=_lib.PREC_BF16X3)),
                                       ctypes.byref(outs), None, 0, None) == _lib.DQB_ERR_UNSUPPORTED
    # a workspace below the size query is refused before anything runs
    assert lib.dqb_mesolve_dense_large(ctypes.byref(p), ctypes.byref(_opts()), ctypes.byref(outs),
                                       1, 16, None) == _lib.DQB_ERR_WORKSPACE_TOO_SMALL
    assert np.int32(_lib.DQB_ERR_WORKSPACE_TOO_SMALL) == 3
