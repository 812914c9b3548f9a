"""ctypes binding of libcufhedb_b200.so (the C ABI in include/cufhedb_b200.h).

The engine has no CPU fallback: if the shared library is missing, or no
sm_100 device is present, calls raise instead of computing anything.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcufhedb_b200.so")

OK, ERR_ARG, ERR_NOKEY, ERR_CUDA, ERR_OOM, ERR_DEVICE, ERR_UNSUPPORTED = range(7)
FP64, SPLIT32, SPLIT32_TC = 0, 1, 2
KSK10, KSK20, KSK21 = 10, 20, 21
GEN_BK01, GEN_BK02, GEN_KSK10, GEN_KSK20, GEN_KSK21, GEN_ALL = 1, 2, 4, 8, 16, 31
TV_CONST, TV_STAIRCASE, TV_POLY = 0, 1, 2
COMPARE = {"gt": 0, "ge": 1, "lt": 2, "le": 3, "eq": 4}
GATES = {"NAND": 0, "NOR": 1, "XNOR": 2, "AND": 3, "OR": 4, "XOR": 5,
         "ANDNY": 6, "ANDYN": 7, "ORNY": 8, "ORYN": 9}


class CufhedbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cufhedb error {code}: {msg}")
        self.code = code


class TestVec(C.Structure):
    _fields_ = [("kind", C.c_int), ("pad_bits", C.c_int), ("value", C.c_uint64), ("poly", C.c_void_p)]


_vp, _i32, _u32, _u64 = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64


class Query(C.Structure):
    """cufhedb_query: one filter query of a queue (cufhedb_queue_run)"""
    _fields_ = [("level", C.c_int), ("op", C.c_int), ("plain_bits", C.c_uint32), ("logic", C.c_int),
                ("rows", C.c_int), ("c1", C.c_void_p), ("c2", C.c_void_p), ("out", C.c_void_p)]

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "cufhedb_abi_version": [],
    "cufhedb_last_error": [],
    "cufhedb_ctx_create": [C.POINTER(_vp), _i32],
    "cufhedb_ctx_destroy": [_vp],
    "cufhedb_ctx_num_sms": [_vp],
    "cufhedb_sync": [_vp, _vp],
    "cufhedb_load_bkfft_lvl01": [_vp, _vp],
    "cufhedb_load_bk_lvl01": [_vp, _vp],
    "cufhedb_load_ksk": [_vp, _i32, _vp],
    "cufhedb_load_bk_lvl02": [_vp, _vp],
    "cufhedb_load_bkfft_lvl02": [_vp, _vp],
    "cufhedb_export_bk_lvl02": [_vp, _vp],
    "cufhedb_pbs_lvl02": [_vp, _vp, _vp, _i32, C.POINTER(TestVec), _vp],
    "cufhedb_trgsw_prepare_lvl2": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_trgswfft_prepare_lvl2": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_extprod_lvl2": [_vp, _vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_twist_ifft_lvl2": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_twist_fft_lvl2": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_keygen": [_vp, _u64, C.c_uint],
    "cufhedb_export_bk_lvl01": [_vp, _vp],
    "cufhedb_export_ksk_rows": [_vp, _i32, _vp, _i32, _vp],
    "cufhedb_secret_keys": [_u64, _vp, _vp, _vp],
    "cufhedb_encrypt_lvl1": [_vp, _u64, _u64, _u64, _vp, _vp, _i32, _vp],
    "cufhedb_encrypt_lvl2": [_vp, _u64, _u64, _u64, _vp, _vp, _i32, _vp],
    "cufhedb_phase_lvl1": [_vp, _vp, _vp, _vp, _i32, _vp],
    "cufhedb_autotune_pbs01": [_vp, _i32, _vp, _vp],
    "cufhedb_autotune_pbs02": [_vp, _vp],
    "cufhedb_autotune_table": [_vp, _i32, _i32, _vp, _vp],
    "cufhedb_launch_shape": [_vp, _i32, _i32, _i32, _vp],
    "cufhedb_launch_layout": [_vp, _i32, _vp],
    "cufhedb_autotune_save": [_vp, C.c_char_p],
    "cufhedb_autotune_load": [_vp, C.c_char_p],
    "cufhedb_load_keyfile": [_vp, C.c_char_p, _vp],
    "cufhedb_arc_compare": [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _i32, _vp],
    "cufhedb_polymul_lvl1": [_vp, _vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_selftest_wait_timeout": [_vp, C.c_uint32],
    "cufhedb_polymul_lvl2": [_vp, _vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_save_keyfile": [_vp, C.c_char_p, _vp],
    "cufhedb_phase_lvl2": [_vp, _vp, _vp, _vp, _i32, _vp],
    "cufhedb_pbs_lvl01": [_vp, _vp, _vp, _i32, C.POINTER(TestVec), _i32, _vp],
    "cufhedb_iks": [_vp, _i32, _vp, _vp, _i32, _vp],
    "cufhedb_gate_lvl1": [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_gate_lvl1_noalloc": [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_trgsw_prepare_lvl1": [_vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_trgswfft_prepare_lvl1": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_extprod_lvl1": [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp],
    "cufhedb_extprod_lvl1_host": [_vp, _vp, _vp, _vp, _i32, _i32],
    "cufhedb_twist_ifft_lvl1": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_twist_fft_lvl1": [_vp, _vp, _vp, _i32, _vp],
    "cufhedb_pbs_lvl01_host": [_vp, _vp, _vp, _i32, C.POINTER(TestVec), _i32],
    "cufhedb_gate_lvl1_host": [_vp, _i32, _vp, _vp, _vp, _i32, _i32],
    "cufhedb_measure_fma_peak": [_i32, _i32, C.POINTER(C.c_double)],
    "cufhedb_msb_bootstrap": [_vp, _i32, _i32, _vp, _vp, _i32, _i32, _i32, _vp],
    "cufhedb_ide_bootstrap": [_vp, _i32, _i32, _vp, _vp, _i32, _u32, _i32, _vp],
    "cufhedb_log_to_ari": [_vp, _vp, _vp, _i32, _i32, _vp],
    "cufhedb_log_rescale": [_vp, _vp, _vp, _i32, _u32, _i32, _vp],
    "cufhedb_hom_and": [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp],
    "cufhedb_hom_or": [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp],
    "cufhedb_hom_msb": [_vp, _i32, _vp, _vp, _i32, _u32, _i32, _i32, _vp],
    "cufhedb_compare": [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _u32, _i32, _i32, _vp],
    "cufhedb_queue_run": [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp],
    "cufhedb_queue_plan": [_vp, _i32, C.c_double, C.c_double, _i32, _i32, _vp, _vp, _vp],
    "cufhedb_cereal_key_payload": [C.c_char_p, _i32, _vp, _vp],
    "cufhedb_compare_host": [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _u32, _i32, _i32],
    "cufhedb_gate_lvl1_host_multi": [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _i32],
    "cufhedb_compare_host_multi": [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _i32, _u32, _i32, _i32],
    "cufhedb_load_cereal_key": [_vp, C.c_char_p, _i32],
    "cufhedb_graph_begin": [_vp, _vp],
    "cufhedb_graph_end": [_vp, _vp, C.POINTER(_vp)],
    "cufhedb_graph_launch": [_vp, _vp],
    "cufhedb_graph_destroy": [_vp],
}
_RESTYPE = {"cufhedb_last_error": C.c_char_p}

_lock = threading.Lock()
_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load (once) and return the engine library, with signatures set."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise CufhedbError(ERR_UNSUPPORTED, f"{p} is missing: build it with `python -m cufhedb_b200.build`")
        lib = C.CDLL(p)
        for name, args in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, C.c_int)
        _lib = lib
        return lib


def check(rc: int) -> None:
    if rc != OK:
        msg = load().cufhedb_last_error()
        raise CufhedbError(rc, msg.decode() if msg else "")
