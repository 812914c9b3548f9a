"""CPU: the engine library loads, exports every symbol include/*.h declares,
and fails loudly (no CPU fallback) when no sm_100 device is present."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names.update(re.findall(r"CUFHEDB_API\s+[\w\s\*]*?\b(cufhedb_\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "cufhedb_pbs_lvl01" in names and "cufhedb_iks" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from cufhedb_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail("libcufhedb_b200.so not built (python -m cufhedb_b200.build)")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # the python binding covers the same set
    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_abi_version_and_secret_keys_without_gpu():
    import numpy as np
    from cufhedb_b200 import Engine, load
    lib = load()
    assert lib.cufhedb_abi_version() == 1
    s0, s1, s2 = Engine.secret_keys(0x5EED_B200)
    from oracle.oracle import Oracle
    o0, o1, o2 = Oracle().secret_keys(0x5EED_B200)
    assert np.array_equal(s0, o0) and np.array_equal(s1, o1) and np.array_equal(s2, o2)


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cufhedb_b200 import CufhedbError, Engine
    with pytest.raises(CufhedbError):
        Engine(0)


def test_every_context_entry_point_rejects_a_null_context():
    """Every entry point that takes a context validates it before anything
    else: with a null context (and every other argument null or 1, so that no
    empty-batch shortcut applies) it returns CUFHEDB_ERR_ARG with a message and
    touches no device."""
    from cufhedb_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    lib.cufhedb_last_error.restype = ctypes.c_char_p
    checked = 0
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        for name, args in re.findall(r"CUFHEDB_API\s+int\s+(cufhedb_\w+)\s*\(([^)]*)\)", txt):
            params = [a.strip() for a in args.split(",")]
            if not params[0].startswith("cufhedb_ctx *") or name in ("cufhedb_ctx_destroy",):
                continue
            call = []
            for p in params[1:]:
                call.append(None if "*" in p else 1)
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p if a is None else ctypes.c_uint64 for a in call]
            rc = f(None, *call)
            assert rc == _lib.ERR_ARG, (name, rc)
            assert lib.cufhedb_last_error(), name
            checked += 1
    assert checked >= 40
