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
