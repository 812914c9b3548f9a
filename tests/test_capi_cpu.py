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
