"""Host-side mirror of the engine for Python callers (tests, benchmarks).

``Engine`` owns one context (``cufhedb_ctx``) on one device.  Device buffers
are torch CUDA tensors used as raw storage: 32-bit torus words live in
``torch.int32`` tensors and 64-bit ones in ``torch.int64`` tensors, bit for
bit (torch is only the allocator and stream provider here).  Host buffers are
numpy arrays of ``uint32`` / ``uint64`` / ``float64``.

Sizes follow TFHEpp (thirdparty/TFHEpp/include/params/128bit.hpp:7-83).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

N0, N1, L1, N2, L2 = 672, 1024, 3, 2048, 4
MU1 = 1 << 29
BK01_SHAPE = (N0, 2 * L1, 2, N1)


def _ptr(t) -> int:
    """Device or host address of a torch tensor or numpy array."""
    if isinstance(t, np.ndarray):
        if not t.flags["C_CONTIGUOUS"]:
            raise ValueError("numpy buffers must be C-contiguous")
        return t.ctypes.data
    if not t.is_contiguous():
        raise ValueError("tensors must be contiguous")
    return t.data_ptr()


def _stream(stream) -> int | None:
    if stream is None:
        try:
            import torch
            return torch.cuda.current_stream().cuda_stream
        except Exception:
            return None
    return getattr(stream, "cuda_stream", stream)


def testvec_const(mu: int) -> _lib.TestVec:
    return _lib.TestVec(_lib.TV_CONST, 0, mu & 0xFFFFFFFFFFFFFFFF, None)


def testvec_staircase(scale_bits: int, pad_bits: int = 6) -> _lib.TestVec:
    return _lib.TestVec(_lib.TV_STAIRCASE, pad_bits, scale_bits, None)


def testvec_poly(dev_tensor) -> _lib.TestVec:
    return _lib.TestVec(_lib.TV_POLY, 0, 0, C.c_void_p(_ptr(dev_tensor)))


class Engine:
    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.cufhedb_ctx_create(C.byref(h), device))
        self.ctx = h
        self.device = device

    def close(self):
        if self.ctx:
            self.lib.cufhedb_ctx_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_sms(self) -> int:
        return self.lib.cufhedb_ctx_num_sms(self.ctx)

    def sync(self, stream=None):
        check(self.lib.cufhedb_sync(self.ctx, _stream(stream)))

    # ---- keys ----------------------------------------------------------------
    def keygen(self, seed: int, flags: int = _lib.GEN_ALL):
        check(self.lib.cufhedb_keygen(self.ctx, seed, flags))

    def load_bkfft_lvl01(self, bkfft: np.ndarray):
        bkfft = np.ascontiguousarray(bkfft, np.float64)
        assert bkfft.size == N0 * 2 * L1 * 2 * N1
        check(self.lib.cufhedb_load_bkfft_lvl01(self.ctx, _ptr(bkfft)))

    def load_bk_lvl01(self, bk: np.ndarray):
        bk = np.ascontiguousarray(bk, np.uint32)
        assert bk.size == N0 * 2 * L1 * 2 * N1
        check(self.lib.cufhedb_load_bk_lvl01(self.ctx, _ptr(bk)))

    def load_ksk(self, kind: int, ksk: np.ndarray):
        ksk = np.ascontiguousarray(ksk, np.uint32)
        check(self.lib.cufhedb_load_ksk(self.ctx, kind, _ptr(ksk)))

    def load_keyfile(self, path: str) -> np.ndarray:
        """load the lvl01 bootstrapping key and lvl10 key-switching key from a
        key file in the reference's raw layout; returns the stored lvl1 secret key"""
        sk = np.zeros(N1, np.uint32)
        check(self.lib.cufhedb_load_keyfile(self.ctx, path.encode(), _ptr(sk)))
        return sk

    def save_keyfile(self, path: str, sk=None):
        skp = None if sk is None else _ptr(np.ascontiguousarray(sk, np.uint32))
        check(self.lib.cufhedb_save_keyfile(self.ctx, path.encode(), skp))

    CEREAL = {"bkfft01": 1, "bkfft02": 2, "ksk10": 10, "ksk20": 20, "ksk21": 21}

    def load_cereal_key(self, path: str, kind: str):
        """a key from a TFHEpp cereal archive (the reference's serialize.cpp files)"""
        check(self.lib.cufhedb_load_cereal_key(self.ctx, path.encode(), self.CEREAL[kind]))

    def export_bk_lvl01(self) -> np.ndarray:
        out = np.zeros(BK01_SHAPE, np.uint32)
        check(self.lib.cufhedb_export_bk_lvl01(self.ctx, _ptr(out)))
        return out

    def export_ksk_rows(self, kind: int, rows) -> np.ndarray:
        rows = np.ascontiguousarray(rows, np.uint64)
        width = N1 + 1 if kind == 21 else N0 + 1
        out = np.zeros((rows.size, width), np.uint32)
        check(self.lib.cufhedb_export_ksk_rows(self.ctx, kind, _ptr(rows), rows.size, _ptr(out)))
        return out

    @staticmethod
    def secret_keys(seed: int):
        lib = _lib.load()
        s0 = np.zeros(N0, np.uint32); s1 = np.zeros(N1, np.uint32); s2 = np.zeros(N2, np.uint64)
        check(lib.cufhedb_secret_keys(seed, _ptr(s0), _ptr(s1), _ptr(s2)))
        return s0, s1, s2

    def encrypt_lvl1(self, seed: int, stream_id: int, idx0: int, msg_dev, out_dev, stream=None):
        B = msg_dev.numel()
        check(self.lib.cufhedb_encrypt_lvl1(self.ctx, seed, stream_id, idx0, _ptr(msg_dev), _ptr(out_dev), B,
                                            _stream(stream)))

    def encrypt_lvl2(self, seed: int, stream_id: int, idx0: int, msg_dev, out_dev, stream=None):
        B = msg_dev.numel()
        check(self.lib.cufhedb_encrypt_lvl2(self.ctx, seed, stream_id, idx0, _ptr(msg_dev), _ptr(out_dev), B,
                                            _stream(stream)))

    def autotune_pbs01(self, precision: int = _lib.FP64):
        """time one full pass of each lvl01 launch shape (7, 8 and 4
        ciphertexts per CTA); later launches pick the shape with the least
        passes x pass time for their batch.  Returns (ms7, ms8)."""
        a, b = C.c_float(0.0), C.c_float(0.0)
        check(self.lib.cufhedb_autotune_pbs01(self.ctx, precision, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune_pbs02(self):
        """time one full pass of each lvl02 launch shape (3, 2, 1 per CTA);
        returns the three pass times"""
        ms = (C.c_float * 3)()
        check(self.lib.cufhedb_autotune_pbs02(self.ctx, ms))
        return list(ms)

    def autotune_table(self, level: int, precision: int = _lib.FP64):
        """{shape: pass time (ms)} of a level's launch shapes in this context"""
        shapes, ms = (C.c_int * 3)(), (C.c_float * 3)()
        n = self.lib.cufhedb_autotune_table(self.ctx, level, precision, shapes, ms)
        if n != 3:
            check(n)
        return {int(w): float(t) for w, t in zip(shapes, ms)}

    def launch_shape(self, level: int, precision: int, B: int) -> int:
        """ciphertexts per CTA a launch of B bootstraps would use now"""
        w = C.c_int(0)
        check(self.lib.cufhedb_launch_shape(self.ctx, level, precision, B, C.byref(w)))
        return w.value

    def launch_layout(self, B: int) -> str:
        """stage-1 layout a split32 launch of B bootstraps would use now:
        "cuda-core" or "tensor-core" """
        tc = C.c_int(0)
        check(self.lib.cufhedb_launch_layout(self.ctx, B, C.byref(tc)))
        return "tensor-core" if tc.value else "cuda-core"

    def autotune_save(self, path: str):
        check(self.lib.cufhedb_autotune_save(self.ctx, path.encode()))

    def autotune_load(self, path: str) -> bool:
        """restore pass times saved for this device and parameter set; False
        (and nothing changed) when the file is missing or made for another"""
        import os
        if not os.path.exists(path):
            return False
        return self.lib.cufhedb_autotune_load(self.ctx, path.encode()) == 0

    def autotune(self, path: str | None = None, levels=(1, 2)):
        """the persisted launch-shape table: loaded from `path` when it was made
        for this device and parameter set, else measured for every loaded key
        (lvl01 on both precisions, lvl02) and saved to `path`.  Returns
        {"loaded": bool, "pbs01_fp64": {...}, "pbs01_split32": {...}, "pbs01_split32tc": {...},
        "pbs02": {...}}"""
        loaded = bool(path) and self.autotune_load(path)
        if not loaded:
            if 1 in levels:
                self.autotune_pbs01(_lib.FP64)
                self.autotune_pbs01(_lib.SPLIT32)
                self.autotune_pbs01(_lib.SPLIT32_TC)
            if 2 in levels:
                self.autotune_pbs02()
            if path:
                self.autotune_save(path)
        return {"loaded": loaded, "pbs01_fp64": self.autotune_table(1, _lib.FP64),
                "pbs01_split32": self.autotune_table(1, _lib.SPLIT32),
                "pbs01_split32tc": self.autotune_table(1, _lib.SPLIT32_TC), "pbs02": self.autotune_table(2, _lib.FP64)}

    def phase_lvl1(self, ct_dev, phase_dev, key_dev=None, stream=None):
        """decryption phases b - <a, s1> of lvl1 TLWEs (key: device words, or the key set's)"""
        B = ct_dev.numel() // (N1 + 1)
        check(self.lib.cufhedb_phase_lvl1(self.ctx, _ptr(ct_dev), _ptr(key_dev) if key_dev is not None else None,
                                          _ptr(phase_dev), B, _stream(stream)))

    def phase_lvl2(self, ct_dev, phase_dev, key_dev=None, stream=None):
        B = ct_dev.numel() // (N2 + 1)
        check(self.lib.cufhedb_phase_lvl2(self.ctx, _ptr(ct_dev), _ptr(key_dev) if key_dev is not None else None,
                                          _ptr(phase_dev), B, _stream(stream)))

    # ---- batched device operations ---------------------------------------------
    def pbs_lvl01(self, in_dev, out_dev, tv: _lib.TestVec, precision: int = _lib.FP64, stream=None):
        B = in_dev.numel() // (N0 + 1)
        check(self.lib.cufhedb_pbs_lvl01(self.ctx, _ptr(in_dev), _ptr(out_dev), B, C.byref(tv), precision,
                                         _stream(stream)))

    def iks(self, kind: int, in_dev, out_dev, stream=None):
        width = N1 + 1 if kind == 10 else N2 + 1
        B = in_dev.numel() // width
        check(self.lib.cufhedb_iks(self.ctx, kind, _ptr(in_dev), _ptr(out_dev), B, _stream(stream)))

    def gate_lvl1(self, gate: str, ca_dev, cb_dev, out_dev, precision: int = _lib.FP64, stream=None):
        B = ca_dev.numel() // (N1 + 1)
        check(self.lib.cufhedb_gate_lvl1(self.ctx, _lib.GATES[gate], _ptr(ca_dev), _ptr(cb_dev), _ptr(out_dev), B,
                                         precision, _stream(stream)))

    def gate_lvl1_noalloc(self, gate: str, ca_dev, cb_dev, out_dev, precision: int = _lib.FP64, stream=None):
        """Same result as gate_lvl1 without any device allocation: at most
        1,024 gates per call, one shared per-device intermediate (calls that
        overlap on the GPU race)."""
        B = ca_dev.numel() // (N1 + 1)
        check(self.lib.cufhedb_gate_lvl1_noalloc(self.ctx, _lib.GATES[gate], _ptr(ca_dev), _ptr(cb_dev),
                                                 _ptr(out_dev), B, precision, _stream(stream)))

    def trgsw_prepare_lvl1(self, trgsw_dev, out_dev, precision: int = _lib.FP64, stream=None):
        """integer TRGSWs (B x 6 x 2 x 1024 words) -> prepared frequency-domain
        TRGSWs (B x 98,304 bytes, e.g. a float64 tensor of B x 12,288)"""
        B = trgsw_dev.numel() // (2 * L1 * 2 * N1)
        check(self.lib.cufhedb_trgsw_prepare_lvl1(self.ctx, _ptr(trgsw_dev), _ptr(out_dev), B, precision,
                                                  _stream(stream)))

    def trgswfft_prepare_lvl1(self, trgswfft_dev, out_dev, stream=None):
        B = trgswfft_dev.numel() // (2 * L1 * 2 * N1)
        check(self.lib.cufhedb_trgswfft_prepare_lvl1(self.ctx, _ptr(trgswfft_dev), _ptr(out_dev), B,
                                                     _stream(stream)))

    def extprod_lvl1(self, trlwe_dev, trgsw_prepared, out_dev, shared: bool = False, precision: int = _lib.FP64,
                     stream=None):
        B = trlwe_dev.numel() // (2 * N1)
        check(self.lib.cufhedb_extprod_lvl1(self.ctx, _ptr(trlwe_dev), _ptr(trgsw_prepared), _ptr(out_dev), B,
                                            int(shared), precision, _stream(stream)))

    def extprod_lvl1_host(self, trlwe: np.ndarray, trgswfft: np.ndarray, shared: bool = False) -> np.ndarray:
        trlwe = np.ascontiguousarray(trlwe, np.uint32).reshape(-1, 2, N1)
        trgswfft = np.ascontiguousarray(trgswfft, np.float64)
        out = np.zeros_like(trlwe)
        check(self.lib.cufhedb_extprod_lvl1_host(self.ctx, _ptr(trlwe), _ptr(trgswfft), _ptr(out), trlwe.shape[0],
                                                 int(shared)))
        return out

    # ---- lvl2 (64-bit torus, N = 2048), FP64 -----------------------------------
    def load_bk_lvl02(self, bk: np.ndarray):
        bk = np.ascontiguousarray(bk, np.uint64)
        check(self.lib.cufhedb_load_bk_lvl02(self.ctx, _ptr(bk)))

    def load_bkfft_lvl02(self, bkfft: np.ndarray):
        bkfft = np.ascontiguousarray(bkfft, np.float64)
        check(self.lib.cufhedb_load_bkfft_lvl02(self.ctx, _ptr(bkfft)))

    def export_bk_lvl02(self) -> np.ndarray:
        out = np.zeros((N0, 2 * L2, 2, N2), np.uint64)
        check(self.lib.cufhedb_export_bk_lvl02(self.ctx, _ptr(out)))
        return out

    def pbs_lvl02(self, in_dev, out_dev, tv: _lib.TestVec, stream=None):
        B = in_dev.numel() // (N0 + 1)
        check(self.lib.cufhedb_pbs_lvl02(self.ctx, _ptr(in_dev), _ptr(out_dev), B, C.byref(tv), _stream(stream)))

    def trgsw_prepare_lvl2(self, trgsw_dev, out_dev, stream=None):
        B = trgsw_dev.numel() // (2 * L2 * 2 * N2)
        check(self.lib.cufhedb_trgsw_prepare_lvl2(self.ctx, _ptr(trgsw_dev), _ptr(out_dev), B, _stream(stream)))

    def trgswfft_prepare_lvl2(self, trgswfft_dev, out_dev, stream=None):
        B = trgswfft_dev.numel() // (2 * L2 * 2 * N2)
        check(self.lib.cufhedb_trgswfft_prepare_lvl2(self.ctx, _ptr(trgswfft_dev), _ptr(out_dev), B,
                                                     _stream(stream)))

    def extprod_lvl2(self, trlwe_dev, trgsw_prepared, out_dev, shared: bool = False, stream=None):
        B = trlwe_dev.numel() // (2 * N2)
        check(self.lib.cufhedb_extprod_lvl2(self.ctx, _ptr(trlwe_dev), _ptr(trgsw_prepared), _ptr(out_dev), B,
                                            int(shared), _stream(stream)))

    def twist_ifft_lvl2(self, in_dev, out_dev, stream=None):
        B = in_dev.numel() // N2
        check(self.lib.cufhedb_twist_ifft_lvl2(self.ctx, _ptr(in_dev), _ptr(out_dev), B, _stream(stream)))

    def twist_fft_lvl2(self, in_dev, out_dev, stream=None):
        B = in_dev.numel() // N2
        check(self.lib.cufhedb_twist_fft_lvl2(self.ctx, _ptr(in_dev), _ptr(out_dev), B, _stream(stream)))

    def twist_ifft_lvl1(self, in_dev, out_dev, stream=None):
        B = in_dev.numel() // N1
        check(self.lib.cufhedb_twist_ifft_lvl1(self.ctx, _ptr(in_dev), _ptr(out_dev), B, _stream(stream)))

    def twist_fft_lvl1(self, in_dev, out_dev, stream=None):
        B = in_dev.numel() // N1
        check(self.lib.cufhedb_twist_fft_lvl1(self.ctx, _ptr(in_dev), _ptr(out_dev), B, _stream(stream)))

    # ---- operator layer (cuHEDB operators over batches of rows) --------------------
    @staticmethod
    def _rows(t, level):
        return t.numel() // ((N1 + 1) if level == 1 else (N2 + 1))

    def msb_bootstrap(self, in_level, out_level, in_dev, out_dev, logic=True, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_msb_bootstrap(self.ctx, in_level, out_level, _ptr(in_dev), _ptr(out_dev),
                                             self._rows(in_dev, in_level), int(logic), precision, _stream(stream)))

    def ide_bootstrap(self, in_level, out_level, in_dev, out_dev, scale_bits, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_ide_bootstrap(self.ctx, in_level, out_level, _ptr(in_dev), _ptr(out_dev),
                                             self._rows(in_dev, in_level), scale_bits, precision, _stream(stream)))

    def log_to_ari(self, in_dev, out_dev, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_log_to_ari(self.ctx, _ptr(in_dev), _ptr(out_dev), self._rows(in_dev, 1), precision,
                                          _stream(stream)))

    def hom_and(self, ca, cb, out, logic=True, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_hom_and(self.ctx, _ptr(ca), _ptr(cb), _ptr(out), self._rows(ca, 1), int(logic),
                                       precision, _stream(stream)))

    def hom_or(self, ca, cb, out, logic=True, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_hom_or(self.ctx, _ptr(ca), _ptr(cb), _ptr(out), self._rows(ca, 1), int(logic),
                                      precision, _stream(stream)))

    def hom_msb(self, in_level, in_dev, out_dev, plain_bits, logic=True, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_hom_msb(self.ctx, in_level, _ptr(in_dev), _ptr(out_dev), self._rows(in_dev, in_level),
                                       plain_bits, int(logic), precision, _stream(stream)))

    def compare(self, op: str, level: int, c1, c2, out, plain_bits, logic=True, precision=_lib.FP64, stream=None):
        check(self.lib.cufhedb_compare(self.ctx, _lib.COMPARE[op], level, _ptr(c1), _ptr(c2), _ptr(out),
                                       self._rows(c1, level), plain_bits, int(logic), precision, _stream(stream)))

    def queue_run(self, queries, precision: int = _lib.FP64, max_batch_rows: int = 16384, nstreams: int = 2):
        """Run a queue of filter queries through the native scheduler.
        queries: list of (op, level, c1_dev, c2_dev, out_dev, plain_bits, logic)
        with rows taken from out_dev.  Returns (latency_ms per query, total_ms)."""
        n = len(queries)
        arr = (_lib.Query * max(n, 1))()
        for i, (op, level, c1, c2, out, pb, logic) in enumerate(queries):
            arr[i] = _lib.Query(level, _lib.COMPARE[op] if isinstance(op, str) else op, pb, int(logic),
                                out.numel() // (N1 + 1), _ptr(c1), _ptr(c2), _ptr(out))
        lat = (C.c_float * max(n, 1))()
        total = C.c_float(0.0)
        check(self.lib.cufhedb_queue_run(self.ctx, arr, n, precision, max_batch_rows, nstreams, lat, C.byref(total)))
        return [float(x) for x in lat[:n]], float(total.value)

    def polymul_lvl1(self, a_dev, m_fd_dev, out_dev, shared: bool = True, stream=None):
        """negacyclic products a_i * m, m in TFHEpp's frequency-domain layout"""
        B = a_dev.numel() // N1
        check(self.lib.cufhedb_polymul_lvl1(self.ctx, _ptr(a_dev), _ptr(m_fd_dev), _ptr(out_dev), B, int(shared),
                                            _stream(stream)))

    def polymul_lvl2(self, a_dev, m_fd_dev, out_dev, shared: bool = True, stream=None):
        B = a_dev.numel() // N2
        check(self.lib.cufhedb_polymul_lvl2(self.ctx, _ptr(a_dev), _ptr(m_fd_dev), _ptr(out_dev), B, int(shared),
                                            _stream(stream)))

    def selftest_wait_timeout(self, polls: int = 4096) -> int:
        """run the bounded-wait self-test; returns the raw status (ERR_DEVICE
        when the expired wait was recorded and reported, as it should be)"""
        return self.lib.cufhedb_selftest_wait_timeout(self.ctx, polls)

    ARC_OPS = {"gt": 0, "lt": 1, "eq": 2, "lt_strict": 3}

    def arc_compare(self, op: str, trlwe_dev, trgsw_prepared, out_dev, digits: int, precision=_lib.FP64,
                    stream=None):
        """ArcEDB comparison of B rows of `digits` radix-1024 digits (digit-major layouts)"""
        B = trlwe_dev.numel() // (digits * 2 * N1)
        check(self.lib.cufhedb_arc_compare(self.ctx, self.ARC_OPS[op], _ptr(trlwe_dev), _ptr(trgsw_prepared),
                                           _ptr(out_dev), B, digits, precision, _stream(stream)))

    def graph_begin(self, stream):
        check(self.lib.cufhedb_graph_begin(self.ctx, _stream(stream)))

    def graph_end(self, stream):
        g = C.c_void_p()
        check(self.lib.cufhedb_graph_end(self.ctx, _stream(stream), C.byref(g)))
        return g

    def graph_launch(self, graph, stream):
        check(self.lib.cufhedb_graph_launch(graph, _stream(stream)))

    def graph_destroy(self, graph):
        check(self.lib.cufhedb_graph_destroy(graph))

    # ---- host-buffer entry points --------------------------------------------------
    def pbs_lvl01_host(self, in_lvl0: np.ndarray, tv: _lib.TestVec, precision: int = _lib.FP64) -> np.ndarray:
        in_lvl0 = np.ascontiguousarray(in_lvl0, np.uint32).reshape(-1, N0 + 1)
        out = np.zeros((in_lvl0.shape[0], N1 + 1), np.uint32)
        check(self.lib.cufhedb_pbs_lvl01_host(self.ctx, _ptr(in_lvl0), _ptr(out), in_lvl0.shape[0], C.byref(tv),
                                              precision))
        return out

    def gate_lvl1_host(self, gate: str, ca: np.ndarray, cb: np.ndarray, precision: int = _lib.FP64,
                       out: np.ndarray | None = None) -> np.ndarray:
        ca = np.ascontiguousarray(ca, np.uint32).reshape(-1, N1 + 1)
        cb = np.ascontiguousarray(cb, np.uint32).reshape(-1, N1 + 1)
        if out is None:
            out = np.zeros_like(ca)
        check(self.lib.cufhedb_gate_lvl1_host(self.ctx, _lib.GATES[gate], _ptr(ca), _ptr(cb), _ptr(out),
                                              ca.shape[0], precision))
        return out


def _ctx_array(engines):
    arr = (C.c_void_p * len(engines))()
    for i, e in enumerate(engines):
        arr[i] = e.ctx
    return arr


def queue_plan(queries, t01_ms: float, t02_ms: float, max_batch_rows: int = 16384, nstreams: int = 2):
    """The native queue scheduler's plan (host only, no device): queries is a
    list of (op, level, rows, plain_bits, logic); returns (batch of each
    query, stream of each batch), batches numbered in run order."""
    lib = _lib.load()
    n = len(queries)
    arr = (_lib.Query * max(n, 1))()
    for i, (op, level, rows, pb, logic) in enumerate(queries):
        arr[i] = _lib.Query(level, _lib.COMPARE[op] if isinstance(op, str) else op, pb, int(logic), rows,
                            None, None, None)
    batch_of = (C.c_int * max(n, 1))()
    stream_of = (C.c_int * max(n, 1))()
    nb = C.c_int(0)
    check(lib.cufhedb_queue_plan(arr, n, float(t01_ms), float(t02_ms), max_batch_rows, nstreams, batch_of,
                                 stream_of, C.byref(nb)))
    return [int(x) for x in batch_of[:n]], [int(x) for x in stream_of[:nb.value]]


def compare_host(engine: Engine, op: str, level: int, c1: np.ndarray, c2: np.ndarray, plain_bits: int,
                 logic: bool = True, precision: int = _lib.FP64) -> np.ndarray:
    """cufhedb_compare on host arrays (B x (N+1) words of `level`); returns B lvl1 TLWEs"""
    dt = np.uint32 if level == 1 else np.uint64
    width = (N1 if level == 1 else N2) + 1
    c1 = np.ascontiguousarray(c1, dt).reshape(-1, width)
    c2 = np.ascontiguousarray(c2, dt).reshape(-1, width)
    out = np.zeros((c1.shape[0], N1 + 1), np.uint32)
    check(engine.lib.cufhedb_compare_host(engine.ctx, _lib.COMPARE[op], level, _ptr(c1), _ptr(c2), _ptr(out),
                                          c1.shape[0], plain_bits, int(logic), precision))
    return out


def gate_lvl1_host_multi(engines, gate: str, ca: np.ndarray, cb: np.ndarray, precision: int = _lib.FP64):
    """HomGate over host arrays, rows sharded over the engines' contexts
    (one per GPU), one host thread each"""
    ca = np.ascontiguousarray(ca, np.uint32).reshape(-1, N1 + 1)
    cb = np.ascontiguousarray(cb, np.uint32).reshape(-1, N1 + 1)
    out = np.zeros_like(ca)
    lib = engines[0].lib
    check(lib.cufhedb_gate_lvl1_host_multi(_ctx_array(engines), len(engines), _lib.GATES[gate], _ptr(ca), _ptr(cb),
                                           _ptr(out), ca.shape[0], precision))
    return out


def compare_host_multi(engines, op: str, level: int, c1: np.ndarray, c2: np.ndarray, plain_bits: int,
                       logic: bool = True, precision: int = _lib.FP64) -> np.ndarray:
    """compare_host with the rows sharded over the engines' contexts"""
    dt = np.uint32 if level == 1 else np.uint64
    width = (N1 if level == 1 else N2) + 1
    c1 = np.ascontiguousarray(c1, dt).reshape(-1, width)
    c2 = np.ascontiguousarray(c2, dt).reshape(-1, width)
    out = np.zeros((c1.shape[0], N1 + 1), np.uint32)
    lib = engines[0].lib
    check(lib.cufhedb_compare_host_multi(_ctx_array(engines), len(engines), _lib.COMPARE[op], level, _ptr(c1),
                                         _ptr(c2), _ptr(out), c1.shape[0], plain_bits, int(logic), precision))
    return out
