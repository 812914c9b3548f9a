"""GPU: the C++ drop-in headers (include/cufhedb_b200/cuhedb_gpu.hpp and
comparable_gpu.hpp) used the way the reference's own GPU programs use its
cuHEDB / cuARCEDB / cufft layer --
TFHEpp-generated keys, cufftlvl1/2.LoadBK, cuHEDB:: operators on TFHEpp
ciphertexts -- checked against plaintext and the reference's CPU operators.

The program (tests/cpp/dropin_check.cpp) is compiled where the reference's
headers are (``make -C tests/cpp``, run by the package build step) and runs
from its built binary."""
from __future__ import annotations

import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_build", "dropin_check")
ARC_BIN = os.path.join(HERE, "_build", "arc_dropin_check")


def _run(*args, timeout, binary=BIN):
    if not os.path.exists(binary):
        pytest.skip(f"tests/_build/{os.path.basename(binary)} is built only where the reference's TFHEpp headers are")
    r = subprocess.run([binary, *args], capture_output=True, text=True, timeout=timeout)
    print(r.stdout[-6000:])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "FAIL" not in r.stdout


def test_dropin_header_lvl1():
    _run(timeout=900)


def test_dropin_header_lvl2():
    _run("--lvl2", timeout=1500)


def test_dropin_header_arcedb():
    """include/cufhedb_b200/comparable_gpu.hpp: the cuARCEDB:: comparisons,
    HomAND / HomOR, lift_and_and and PolyMul_st, as test/Arc_Query/comparable.cu
    uses them"""
    _run(timeout=900, binary=ARC_BIN)
