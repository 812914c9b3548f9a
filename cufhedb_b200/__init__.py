"""cufhedb_b200: B200-native (sm_100a) TFHE programmable-bootstrapping engine.

The batched PBS / key-switch / external-product path of cuFHEDB's GPU layer
(src/cuHEDB/) re-built for Blackwell, behind a C ABI
(include/cufhedb_b200.h, built into libcufhedb_b200.so).  This package is the
Python host mirror of that ABI; the C++ drop-in for cuFHEDB's own operator
API is include/cufhedb_b200/cuhedb_gpu.hpp.
"""
from ._lib import (FP64, SPLIT32, SPLIT32_TC, KSK10, KSK20, KSK21, GEN_ALL, GEN_BK01, GEN_BK02, GEN_KSK10, GEN_KSK20,
                   GEN_KSK21, GATES, CufhedbError, load)
from .engine import (Engine, N0, N1, N2, L1, L2, MU1, testvec_const, testvec_poly, testvec_staircase)

__all__ = [
    "Engine", "CufhedbError", "load", "FP64", "SPLIT32", "SPLIT32_TC", "KSK10", "KSK20", "KSK21", "GEN_ALL", "GEN_BK01",
    "GEN_BK02", "GEN_KSK10", "GEN_KSK20", "GEN_KSK21", "GATES", "N0", "N1", "N2", "L1", "L2", "MU1",
    "testvec_const", "testvec_poly", "testvec_staircase",
]
