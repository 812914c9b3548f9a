"""TEST ORACLE -- not part of the product.

ctypes bindings for the two CPU checkers used by tests/, by
``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg:

* ``Oracle``  -- oracle/liboracle.so, the plain-C restatement of TFHEpp's PBS
  path (oracle/tfhe_oracle.c), including the deterministic key generator whose
  output the GPU key generator reproduces bit for bit;
* ``RefTFHEpp`` -- oracle/_ref/libtfheref.so, the reference's own TFHEpp and
  HEDB CPU code compiled from its sources (oracle/Makefile, target ``ref``).

Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
N0, N1, L1, BG1, N2, L2, BG2 = 672, 1024, 3, 6, 2048, 4, 9
MU1 = 1 << 29

NS_LVL0, NS_LVL1, NS_LVL2 = 113512, 222, 7094

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _sig(lib, name, args, res=None):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res
    return f


class Oracle:
    """The C restatement (oracle/tfhe_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        u64, i64, i32, u32 = C.c_uint64, C.c_int64, C.c_int, C.c_uint32
        self.draw = _sig(L, "orc_draw", [u64, u64, u64], u64)
        self.noise = _sig(L, "orc_noise", [u64, u64, u64, i64], i64)
        self._sk = _sig(L, "orc_secret_keys", [u64, _u32p, _u32p, _u64p])
        self._t32 = _sig(L, "orc_tlwe32_encrypt", [_u32p, i32, u32, _u32p, i64, u64, u64, u64])
        self._t64 = _sig(L, "orc_tlwe64_encrypt", [_u64p, i32, u64, _u64p, i64, u64, u64, u64])
        self._ph32 = _sig(L, "orc_tlwe32_phase", [_u32p, i32, _u32p], u32)
        self._ph64 = _sig(L, "orc_tlwe64_phase", [_u64p, i32, _u64p], u64)
        self._bk01 = _sig(L, "orc_bk01", [u64, _u32p, _u32p, _u32p, i32])
        self._bk02 = _sig(L, "orc_bk02", [u64, _u32p, _u64p, _u64p, i32])
        self._trgsw32 = _sig(L, "orc_trgsw32", [_u32p, u32, _u32p, u64, u64, u64])
        self._trgsw64 = _sig(L, "orc_trgsw64", [_u64p, u64, _u64p, u64, u64, u64])
        self._trlwe32 = _sig(L, "orc_trlwe32_encrypt", [_u32p, _u32p, _u32p, u64, u64, u64])
        self._k10row = _sig(L, "orc_ksk10_row", [u64, _u32p, _u32p, i32, i32, i32, _u32p])
        self._k20row = _sig(L, "orc_ksk20_row", [u64, _u64p, _u32p, i32, i32, i32, _u32p])
        self._k21row = _sig(L, "orc_ksk21_row", [u64, _u64p, _u32p, i32, i32, i32, _u32p])
        self._kfull = _sig(L, "orc_ksk_full", [i32, u64, _u32p, _u32p, _u64p, C.c_void_p, i32])
        self.ksk_words = _sig(L, "orc_ksk_words", [i32], C.c_size_t)
        self._ifft32 = _sig(L, "orc_twist_ifft32", [_f64p, _u32p, i32])
        self._fft32 = _sig(L, "orc_twist_fft32", [_u32p, _f64p, i32])
        self._ifft64 = _sig(L, "orc_twist_ifft64", [_f64p, _u64p, i32])
        self._fft64 = _sig(L, "orc_twist_fft64", [_u64p, _f64p, i32])
        self._dec32 = _sig(L, "orc_decomp32", [_u32p, _u32p, i32])
        self._dec64 = _sig(L, "orc_decomp64", [_u64p, _u64p, i32])
        self._ep32f = _sig(L, "orc_extprod32_fft", [_u32p, _u32p, _f64p])
        self._ep64f = _sig(L, "orc_extprod64_fft", [_u64p, _u64p, _f64p])
        self._ep32x = _sig(L, "orc_extprod32_exact", [_u32p, _u32p, _u32p])
        self._ep64x = _sig(L, "orc_extprod64_exact", [_u64p, _u64p, _u64p])
        self._g32fft = _sig(L, "orc_trgsw32_fft", [_f64p, _u32p])
        self._g64fft = _sig(L, "orc_trgsw64_fft", [_f64p, _u64p])
        self._pbs01 = _sig(L, "orc_pbs01", [_u32p, _u32p, _f64p, _u32p])
        self._pbs01x = _sig(L, "orc_pbs01_exact", [_u32p, _u32p, _u32p, _u32p])
        self._bkxprep = _sig(L, "orc_bk01_exact_prepare", [_f64p, _u32p])
        self._ep32xs = _sig(L, "orc_extprod32_exact_split", [_u32p, _u32p, _f64p, C.POINTER(C.c_double)])
        self._pbs01xb = _sig(L, "orc_pbs01_exact_batch", [_u32p, _u32p, i32, _f64p, _u32p, i32,
                                                           C.POINTER(C.c_double)])
        self._pbs02 = _sig(L, "orc_pbs02", [_u64p, _u32p, _f64p, _u64p])
        self._br01 = _sig(L, "orc_blind_rotate01", [_u32p, _u32p, _f64p, _u32p])
        self._iks10 = _sig(L, "orc_iks10", [_u32p, _u32p, u64, _u32p, _u32p, C.c_void_p])
        self._iks20 = _sig(L, "orc_iks20", [_u32p, _u64p, u64, _u64p, _u32p, C.c_void_p])
        self._iks21 = _sig(L, "orc_iks21", [_u32p, _u64p, u64, _u64p, _u32p, C.c_void_p])
        self._rows = _sig(L, "orc_iks_rows", [i32, C.c_void_p, _u8p])
        self._gp32 = _sig(L, "orc_tv_gpoly32", [_u32p, u32, u32])
        self._gp64 = _sig(L, "orc_tv_gpoly64", [_u64p, u32, u32])
        self._nand = _sig(L, "orc_homnand", [_u32p, _u32p, _u32p, _f64p, u64, _u32p, _u32p, C.c_void_p])
        self.lib = L

    # ---- keys ---------------------------------------------------------------
    def secret_keys(self, seed):
        s0 = np.zeros(N0, np.uint32); s1 = np.zeros(N1, np.uint32); s2 = np.zeros(N2, np.uint64)
        self._sk(seed, s0, s1, s2)
        return s0, s1, s2

    def bk01(self, seed, s0, s1, nthreads=os.cpu_count() or 1):
        bk = np.zeros((N0, 2 * L1, 2, N1), np.uint32)
        self._bk01(seed, s0, s1, bk, nthreads)
        return bk

    def bk02(self, seed, s0, s2, nthreads=os.cpu_count() or 1):
        bk = np.zeros((N0, 2 * L2, 2, N2), np.uint64)
        self._bk02(seed, s0, s2, bk, nthreads)
        return bk

    def trgsw32(self, m0, s1, seed, stream, idx):
        g = np.zeros((2 * L1, 2, N1), np.uint32)
        self._trgsw32(g, m0, s1, seed, stream, idx)
        return g

    def trgsw64(self, m0, s2, seed, stream, idx):
        g = np.zeros((2 * L2, 2, N2), np.uint64)
        self._trgsw64(g, m0, s2, seed, stream, idx)
        return g

    def trlwe32(self, plain, s1, seed, stream, idx):
        out = np.zeros((2, N1), np.uint32)
        self._trlwe32(out, np.ascontiguousarray(plain, np.uint32), s1, seed, stream, idx)
        return out

    # ---- ArcEDB encodings and single-digit comparisons -----------------------
    def arc_trlwe(self, v, s1, seed, stream, idx):
        """exponent_encrypt<Lvl1> (src/ARCEDB/comparison/comparable.h:169-179):
        the TRLWE of mu X^v, v in [0, N)"""
        plain = np.zeros(N1, np.uint32)
        plain[v] = MU1
        return self.trlwe32(plain, s1, seed, stream, idx)

    def arc_trgsw(self, v, s1, seed, stream, idx):
        """exponent_encrypt_rgsw<Lvl1>(is_negative = true) (comparable.h:228-274):
        the TRGSW of X^{-v}; -h_i at coefficient N - v, or +h_i at 0 when v = 0"""
        g = self.trgsw32(0, s1, seed, stream, idx)
        for i in range(L1):
            h = 1 << (32 - (i + 1) * BG1)
            for k in range(2):
                j = N1 - v if v else 0
                g[i + k * L1, k, j] = (int(g[i + k * L1, k, j]) + (-h if v else h)) % 2 ** 32
        return g

    def arc_single(self, op, trlwe, g):
        """greater_than_tfhepp / less_than_tfhepp / equality_tfhepp of one digit
        (comparable.cpp:506-523, 652-666, 623-633) with the exact external
        product; op "lt_strict" uses the test polynomial -1 + X + ... + X^{N-1}."""
        t = self.extprod32_exact(trlwe, g)
        if op == "eq":
            out = sample_extract32(t) * np.uint32(2)
            out[N1] = (int(out[N1]) - MU1) % 2 ** 32
            return out
        p = np.ones(N1, np.uint32)
        if op == "lt_strict":
            p[0] = np.uint32(0xFFFFFFFF)
        out = sample_extract32(np.stack([polymul32(t[0], p), polymul32(t[1], p)]))
        return (np.uint32(0) - out) if op == "gt" else out

    def ksk_row(self, kind, seed, keys, i, j, k):
        s0, s1, s2 = keys
        if kind == 10:
            r = np.zeros(N0 + 1, np.uint32); self._k10row(seed, s1, s0, i, j, k, r)
        elif kind == 20:
            r = np.zeros(N0 + 1, np.uint32); self._k20row(seed, s2, s0, i, j, k, r)
        else:
            r = np.zeros(N1 + 1, np.uint32); self._k21row(seed, s2, s1, i, j, k, r)
        return r

    def ksk_full_into(self, kind, seed, keys, ptr, nthreads=os.cpu_count() or 1):
        s0, s1, s2 = keys
        self._kfull(kind, seed, s0, s1, s2, ptr, nthreads)

    # ---- encryption ---------------------------------------------------------
    def tlwe32(self, m, key, noise_scale, seed, stream, idx):
        n = key.shape[0]
        c = np.zeros(n + 1, np.uint32)
        self._t32(c, n, int(m) & 0xFFFFFFFF, key, noise_scale, seed, stream, idx)
        return c

    def tlwe64(self, m, key, noise_scale, seed, stream, idx):
        n = key.shape[0]
        c = np.zeros(n + 1, np.uint64)
        self._t64(c, n, int(m) & 0xFFFFFFFFFFFFFFFF, key, noise_scale, seed, stream, idx)
        return c

    def phase32(self, c, key):
        return int(self._ph32(np.ascontiguousarray(c, np.uint32), key.shape[0], key))

    def phase64(self, c, key):
        return int(self._ph64(np.ascontiguousarray(c, np.uint64), key.shape[0], key))

    # ---- transforms and products ---------------------------------------------
    def twist_ifft32(self, a):
        out = np.zeros(a.shape[-1], np.float64); self._ifft32(out, np.ascontiguousarray(a, np.uint32), a.shape[-1]); return out

    def twist_fft32(self, v):
        out = np.zeros(v.shape[-1], np.uint32); self._fft32(out, np.ascontiguousarray(v, np.float64), v.shape[-1]); return out

    def twist_ifft64(self, a):
        out = np.zeros(a.shape[-1], np.float64); self._ifft64(out, np.ascontiguousarray(a, np.uint64), a.shape[-1]); return out

    def twist_fft64(self, v):
        out = np.zeros(v.shape[-1], np.uint64); self._fft64(out, np.ascontiguousarray(v, np.float64), v.shape[-1]); return out

    def decomp32(self, poly, d):
        out = np.zeros(N1, np.uint32); self._dec32(out, np.ascontiguousarray(poly, np.uint32), d); return out

    def decomp64(self, poly, d):
        out = np.zeros(N2, np.uint64); self._dec64(out, np.ascontiguousarray(poly, np.uint64), d); return out

    def trgsw32_fft(self, g):
        out = np.zeros((2 * L1, 2, N1), np.float64); self._g32fft(out, np.ascontiguousarray(g, np.uint32)); return out

    def trgsw64_fft(self, g):
        out = np.zeros((2 * L2, 2, N2), np.float64); self._g64fft(out, np.ascontiguousarray(g, np.uint64)); return out

    def extprod32_fft(self, trlwe, gfft):
        r = np.zeros((2, N1), np.uint32); self._ep32f(r, np.ascontiguousarray(trlwe, np.uint32), np.ascontiguousarray(gfft)); return r

    def extprod64_fft(self, trlwe, gfft):
        r = np.zeros((2, N2), np.uint64); self._ep64f(r, np.ascontiguousarray(trlwe, np.uint64), np.ascontiguousarray(gfft)); return r

    def extprod32_exact(self, trlwe, g):
        r = np.zeros((2, N1), np.uint32); self._ep32x(r, np.ascontiguousarray(trlwe, np.uint32), np.ascontiguousarray(g, np.uint32)); return r

    def extprod64_exact(self, trlwe, g):
        r = np.zeros((2, N2), np.uint64); self._ep64x(r, np.ascontiguousarray(trlwe, np.uint64), np.ascontiguousarray(g, np.uint64)); return r

    def bkfft01(self, bk):
        """FFT-domain bootstrapping key [672][6][2][1024] from the integer key."""
        out = np.zeros(bk.shape, np.float64)
        for i in range(bk.shape[0]):
            out[i] = self.trgsw32_fft(bk[i])
        return out

    def pbs01(self, in0, bkfft, tv):
        out = np.zeros(N1 + 1, np.uint32)
        self._pbs01(out, np.ascontiguousarray(in0, np.uint32), bkfft, np.ascontiguousarray(tv, np.uint32))
        return out

    def pbs01_exact(self, in0, bk, tv):
        out = np.zeros(N1 + 1, np.uint32)
        self._pbs01x(out, np.ascontiguousarray(in0, np.uint32), bk, np.ascontiguousarray(tv, np.uint32))
        return out

    def bk01_exact_prepare(self, bk):
        """the integer lvl01 key [672][6][2][1024] in the form the fast exact
        PBS reads: each polynomial split into signed 16-bit limbs, transformed
        ([672][6][2][2][1024] doubles, 132 MB)"""
        bk = np.ascontiguousarray(bk, np.uint32)
        prep = np.zeros((bk.shape[0], bk.shape[1], 2, 2, N1), np.float64)
        self._bkxprep(prep, bk)
        return prep

    def extprod32_exact_split(self, trlwe, prep_trgsw):
        """(exact external product, largest distance of an FFT product from an integer)"""
        res = np.zeros((2, N1), np.uint32)
        dev = C.c_double(0.0)
        self._ep32xs(res, np.ascontiguousarray(trlwe, np.uint32), np.ascontiguousarray(prep_trgsw, np.float64),
                     C.byref(dev))
        return res, dev.value

    def pbs01_exact_batch(self, in0, prep, tv, nthreads=os.cpu_count() or 1):
        """exact lvl01 PBS of n lvl0 ciphertexts on host threads: (n x 1025
        outputs, largest distance of an FFT product from an integer)"""
        in0 = np.ascontiguousarray(in0, np.uint32).reshape(-1, N0 + 1)
        out = np.zeros((in0.shape[0], N1 + 1), np.uint32)
        dev = C.c_double(0.0)
        self._pbs01xb(out, in0, in0.shape[0], prep, np.ascontiguousarray(tv, np.uint32), nthreads, C.byref(dev))
        return out, dev.value

    def pbs02(self, in0, bkfft, tv):
        out = np.zeros(N2 + 1, np.uint64)
        self._pbs02(out, np.ascontiguousarray(in0, np.uint32), bkfft, np.ascontiguousarray(tv, np.uint64))
        return out

    def iks(self, kind, x, seed, keys, ksk_ptr=None):
        s0, s1, s2 = keys
        if kind == 10:
            out = np.zeros(N0 + 1, np.uint32); self._iks10(out, np.ascontiguousarray(x, np.uint32), seed, s1, s0, ksk_ptr)
        elif kind == 20:
            out = np.zeros(N0 + 1, np.uint32); self._iks20(out, np.ascontiguousarray(x, np.uint64), seed, s2, s0, ksk_ptr)
        else:
            out = np.zeros(N1 + 1, np.uint32); self._iks21(out, np.ascontiguousarray(x, np.uint64), seed, s2, s1, ksk_ptr)
        return out

    def iks_rows(self, kind, x):
        n = {10: 1024 * 2 * 1023, 20: 2048 * 2 * 1023, 21: 2048 * 10 * 7}[kind]
        used = np.zeros(n, np.uint8)
        arr = np.ascontiguousarray(x, np.uint32 if kind == 10 else np.uint64)
        self._rows(kind, arr.ctypes.data, used)
        return np.nonzero(used)[0]

    def gpoly32(self, plain_bits, scale_bits):
        tv = np.zeros(N1, np.uint32); self._gp32(tv, plain_bits, scale_bits); return tv

    def gpoly64(self, plain_bits, scale_bits):
        tv = np.zeros(N2, np.uint64); self._gp64(tv, plain_bits, scale_bits); return tv

    def homnand(self, ca, cb, bkfft01, seed, keys, ksk_ptr=None):
        s0, s1, _ = keys
        out = np.zeros(N1 + 1, np.uint32)
        self._nand(out, np.ascontiguousarray(ca, np.uint32), np.ascontiguousarray(cb, np.uint32),
                   bkfft01, seed, s1, s0, ksk_ptr)
        return out


def sample_extract32(trlwe):
    """SampleExtractIndex(index 0) (TFHEpp src/trlwe.cpp:108-118)"""
    a, b = np.asarray(trlwe, np.uint32)
    out = np.empty(N1 + 1, np.uint32)
    out[0] = a[0]
    out[1:N1] = np.uint32(0) - a[:0:-1]
    out[N1] = b[0]
    return out


def polymul32(a, p):
    """negacyclic a * p mod 2^32, exact (TFHEpp PolyMul, include/mulfft.hpp:124-153)"""
    a = np.asarray(a, np.uint64)
    full = np.zeros(2 * len(a), np.uint64)
    for j, pj in enumerate(np.asarray(p, np.uint64)):
        if pj:
            full[j:j + len(a)] += a * pj
    return (full[:len(a)] - full[len(a):]).astype(np.uint32)


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libtfheref.so"))


class RefTFHEpp:
    """The reference's own TFHEpp + HEDB CPU code (oracle/_ref/libtfheref.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "_ref", "libtfheref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = C.CDLL(path)
        vp, i32, u32 = C.c_void_p, C.c_int, C.c_uint32
        _sig(L, "tref_new", [], vp)
        _sig(L, "tref_free", [vp])
        _sig(L, "tref_set_secret", [vp, _u32p, _u32p, _u64p])
        _sig(L, "tref_set_bk01_int", [vp, _u32p])
        _sig(L, "tref_set_bk02_int", [vp, _u64p])
        _sig(L, "tref_get_bkfft01", [vp, _f64p])
        _sig(L, "tref_get_bkfft02", [vp, _f64p])
        _sig(L, "tref_ksk_alloc", [vp, i32], vp)
        _sig(L, "tref_ksk_bytes", [i32], C.c_size_t)
        _sig(L, "tref_twist_ifft_lvl1", [_f64p, _u32p])
        _sig(L, "tref_twist_fft_lvl1", [_u32p, _f64p])
        _sig(L, "tref_twist_ifft_lvl2", [_f64p, _u64p])
        _sig(L, "tref_twist_fft_lvl2", [_u64p, _f64p])
        _sig(L, "tref_decomp_lvl1", [_u32p, _u32p, i32])
        _sig(L, "tref_decomp_lvl2", [_u64p, _u64p, i32])
        _sig(L, "tref_extprod_lvl1", [_u32p, _u32p, _f64p])
        _sig(L, "tref_extprod_lvl2", [_u64p, _u64p, _f64p])
        _sig(L, "tref_pbs01", [vp, _u32p, _u32p, _u32p])
        _sig(L, "tref_pbs02", [vp, _u64p, _u32p, _u64p])
        _sig(L, "tref_iks10", [vp, _u32p, _u32p])
        _sig(L, "tref_iks20", [vp, _u32p, _u64p])
        _sig(L, "tref_iks21", [vp, _u32p, _u64p])
        _sig(L, "tref_homnand", [vp, _u32p, _u32p, _u32p])
        _sig(L, "tref_homnand_batch", [vp, _u32p, _u32p, _u32p, i32, i32])
        _sig(L, "tref_pbs01_batch", [vp, _u32p, _u32p, _u32p, i32, i32])
        _sig(L, "tref_compare_lvl1", [vp, _u32p, _u32p, _u32p, i32, u32, i32])
        _sig(L, "tref_compare_lvl2", [vp, _u32p, _u64p, _u64p, i32, u32, i32])
        _sig(L, "tref_homand", [vp, _u32p, _u32p, _u32p, i32])
        _sig(L, "tref_compare_lvl1_batch", [vp, _u32p, _u32p, _u32p, i32, i32, u32, i32, i32])
        _sig(L, "tref_save_cereal", [vp, i32, C.c_char_p], i32)
        _sig(L, "tref_compare_lvl2_batch", [vp, _u32p, _u64p, _u64p, i32, i32, u32, i32, i32])
        _sig(L, "tref_arc_digit_lvl1", [_u32p, i32, _u32p, _f64p])
        _sig(L, "tref_arc_compare_batch", [vp, _u32p, i32, _u32p, _f64p, i32, i32, i32])
        self.L = L
        self.ctx = L.tref_new()

    def close(self):
        if self.ctx:
            self.L.tref_free(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_secret(self, s0, s1, s2):
        self.L.tref_set_secret(self.ctx, s0, s1, s2)

    def set_bk01(self, bk):
        self.L.tref_set_bk01_int(self.ctx, np.ascontiguousarray(bk, np.uint32))

    def set_bk02(self, bk):
        self.L.tref_set_bk02_int(self.ctx, np.ascontiguousarray(bk, np.uint64))

    def bkfft01(self):
        out = np.zeros((N0, 2 * L1, 2, N1), np.float64); self.L.tref_get_bkfft01(self.ctx, out); return out

    def bkfft02(self):
        out = np.zeros((N0, 2 * L2, 2, N2), np.float64); self.L.tref_get_bkfft02(self.ctx, out); return out

    def ksk_view(self, kind):
        """Zero-initialised full-size key owned by the context, as a numpy view."""
        ptr = self.L.tref_ksk_alloc(self.ctx, kind)
        nbytes = self.L.tref_ksk_bytes(kind)
        buf = (C.c_uint32 * (nbytes // 4)).from_address(ptr)
        width = N1 + 1 if kind == 21 else N0 + 1
        return ptr, np.frombuffer(buf, np.uint32).reshape(-1, width)

    def twist_ifft32(self, a):
        out = np.zeros(N1, np.float64); self.L.tref_twist_ifft_lvl1(out, np.ascontiguousarray(a, np.uint32)); return out

    def twist_fft32(self, v):
        out = np.zeros(N1, np.uint32); self.L.tref_twist_fft_lvl1(out, np.ascontiguousarray(v, np.float64)); return out

    def twist_ifft64(self, a):
        out = np.zeros(N2, np.float64); self.L.tref_twist_ifft_lvl2(out, np.ascontiguousarray(a, np.uint64)); return out

    def twist_fft64(self, v):
        out = np.zeros(N2, np.uint64); self.L.tref_twist_fft_lvl2(out, np.ascontiguousarray(v, np.float64)); return out

    def decomp32(self, poly, d):
        out = np.zeros(N1, np.uint32); self.L.tref_decomp_lvl1(out, np.ascontiguousarray(poly, np.uint32), d); return out

    def decomp64(self, poly, d):
        out = np.zeros(N2, np.uint64); self.L.tref_decomp_lvl2(out, np.ascontiguousarray(poly, np.uint64), d); return out

    def extprod32(self, trlwe, gfft):
        r = np.zeros((2, N1), np.uint32); self.L.tref_extprod_lvl1(r, np.ascontiguousarray(trlwe, np.uint32), np.ascontiguousarray(gfft)); return r

    def extprod64(self, trlwe, gfft):
        r = np.zeros((2, N2), np.uint64); self.L.tref_extprod_lvl2(r, np.ascontiguousarray(trlwe, np.uint64), np.ascontiguousarray(gfft)); return r

    def pbs01(self, in0, tv):
        out = np.zeros(N1 + 1, np.uint32); self.L.tref_pbs01(self.ctx, out, np.ascontiguousarray(in0, np.uint32), np.ascontiguousarray(tv, np.uint32)); return out

    def pbs02(self, in0, tv):
        out = np.zeros(N2 + 1, np.uint64); self.L.tref_pbs02(self.ctx, out, np.ascontiguousarray(in0, np.uint32), np.ascontiguousarray(tv, np.uint64)); return out

    def iks(self, kind, x):
        if kind == 10:
            out = np.zeros(N0 + 1, np.uint32); self.L.tref_iks10(self.ctx, out, np.ascontiguousarray(x, np.uint32))
        elif kind == 20:
            out = np.zeros(N0 + 1, np.uint32); self.L.tref_iks20(self.ctx, out, np.ascontiguousarray(x, np.uint64))
        else:
            out = np.zeros(N1 + 1, np.uint32); self.L.tref_iks21(self.ctx, out, np.ascontiguousarray(x, np.uint64))
        return out

    ARC_DIGIT = {"gt": 0, "lt": 1, "eq": 2, "equal_term": 3}

    def arc_digit(self, op, trlwe, gfft):
        """one digit of the reference's ArcEDB comparison (TFHEpp steps of
        comparable.cpp:506-523 / 652-666 / 623-633)"""
        out = np.zeros(N1 + 1, np.uint32)
        self.L.tref_arc_digit_lvl1(out, self.ARC_DIGIT[op], np.ascontiguousarray(trlwe, np.uint32),
                                   np.ascontiguousarray(gfft, np.float64))
        return out

    def arc_compare_batch(self, op, trlwe, gfft, nthreads=1):
        """the reference's multi-digit ArcEDB comparison of n rows (trlwe
        D x n x 2 x N, gfft D x n TRGSWFFT); needs the lvl01 key and lvl10 key"""
        D, n = trlwe.shape[:2]
        out = np.zeros((n, N1 + 1), np.uint32)
        self.L.tref_arc_compare_batch(self.ctx, out, self.ARC_DIGIT[op], np.ascontiguousarray(trlwe, np.uint32),
                                      np.ascontiguousarray(gfft, np.float64), n, D, nthreads)
        return out

    def homnand(self, ca, cb):
        out = np.zeros(N1 + 1, np.uint32)
        self.L.tref_homnand(self.ctx, out, np.ascontiguousarray(ca, np.uint32), np.ascontiguousarray(cb, np.uint32))
        return out

    def homnand_batch(self, ca, cb, nthreads):
        n = ca.shape[0]
        out = np.zeros((n, N1 + 1), np.uint32)
        self.L.tref_homnand_batch(self.ctx, out, np.ascontiguousarray(ca, np.uint32),
                                  np.ascontiguousarray(cb, np.uint32), n, nthreads)
        return out

    def pbs01_batch(self, in0, tv, nthreads):
        n = in0.shape[0]
        out = np.zeros((n, N1 + 1), np.uint32)
        self.L.tref_pbs01_batch(self.ctx, out, np.ascontiguousarray(in0, np.uint32),
                                np.ascontiguousarray(tv, np.uint32), n, nthreads)
        return out

    def compare_lvl1(self, c1, c2, op, plain_bits, logic=True):
        out = np.zeros(N1 + 1, np.uint32)
        self.L.tref_compare_lvl1(self.ctx, out, np.ascontiguousarray(c1, np.uint32),
                                 np.ascontiguousarray(c2, np.uint32), op, plain_bits, int(logic))
        return out

    def compare_lvl2(self, c1, c2, op, plain_bits, logic=True):
        out = np.zeros(N1 + 1, np.uint32)
        self.L.tref_compare_lvl2(self.ctx, out, np.ascontiguousarray(c1, np.uint64),
                                 np.ascontiguousarray(c2, np.uint64), op, plain_bits, int(logic))
        return out

    def compare_batch(self, level, c1, c2, op, plain_bits, logic=True, nthreads=os.cpu_count() or 1):
        """n rows of HEDB::{greater_than, greater_than_equal, less_than,
        less_than_equal, equal}<level> (op 0..4) on host threads; c1, c2: n x
        (N+1) ciphertexts of that level; returns n lvl1 TLWEs"""
        n = c1.shape[0]
        out = np.zeros((n, N1 + 1), np.uint32)
        if level == 1:
            self.L.tref_compare_lvl1_batch(self.ctx, out, np.ascontiguousarray(c1, np.uint32),
                                           np.ascontiguousarray(c2, np.uint32), n, op, plain_bits, int(logic),
                                           nthreads)
        else:
            self.L.tref_compare_lvl2_batch(self.ctx, out, np.ascontiguousarray(c1, np.uint64),
                                           np.ascontiguousarray(c2, np.uint64), n, op, plain_bits, int(logic),
                                           nthreads)
        return out

    CEREAL = {"bkfft01": 1, "bkfft02": 2, "ksk10": 10, "ksk20": 20, "ksk21": 21}

    def save_cereal(self, kind, path):
        """the context's key as the reference's key tools archive it (cereal
        PortableBinary, EvalKey::serialize_<key>)"""
        rc = self.L.tref_save_cereal(self.ctx, self.CEREAL[kind], path.encode())
        if rc != 0:
            raise RuntimeError(f"tref_save_cereal({kind}) failed")

    def homand(self, ca, cb, logic=True):
        out = np.zeros(N1 + 1, np.uint32)
        self.L.tref_homand(self.ctx, out, np.ascontiguousarray(ca, np.uint32), np.ascontiguousarray(cb, np.uint32), int(logic))
        return out
