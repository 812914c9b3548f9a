"""Generates tests/golden/tfhepp_lvl1.npz and tests/golden/arcedb_lvl1.npz from
the reference's own TFHEpp.

Run in a container that has the reference sources, after `make -C oracle ref`:

    python tests/golden/make_golden.py

Inputs and key material come from the deterministic generator (seed
0x5EEDB200); every output array is computed by the reference's compiled
TFHEpp (oracle/_ref/libtfheref.so), not by the restatement.  The reference
ships no known-answer vectors of its own, so these fixtures pin the oracle
and the engine to the reference's actual behaviour on fixed inputs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import N0, N1, NS_LVL0, NS_LVL1, Oracle, RefTFHEpp  # noqa: E402

SEED = 0x5EED_B200


def main():
    o, r = Oracle(), RefTFHEpp()
    s0, s1, s2 = o.secret_keys(SEED)
    keys = (s0, s1, s2)
    r.set_secret(s0, s1, s2)
    bk = o.bk01(SEED, s0, s1)
    r.set_bk01(bk)
    rng = np.random.default_rng(2024)

    fft_in = rng.integers(0, 2 ** 32, (4, N1), dtype=np.uint64).astype(np.uint32)
    fft_in[0, :4] = [0, 1, 0xFFFFFFFF, 0x80000000]
    fft_out = np.stack([r.twist_ifft32(a) for a in fft_in])
    fft_back = np.stack([r.twist_fft32(v) for v in fft_out])
    dec = [np.stack([r.decomp32(a, d) for a in fft_in]) for d in range(3)]

    iks_in = np.stack([o.tlwe32(int(m) << 29, s1, NS_LVL1, SEED, 0x41, i)
                       for i, m in enumerate(rng.integers(0, 8, 4))])
    _, view = r.ksk_view(10)
    for x in iks_in:
        for row in o.iks_rows(10, x):
            i, rem = divmod(int(row), 2 * 1023)
            j, k = divmod(rem, 1023)
            view[row] = o.ksk_row(10, SEED, keys, i, j, k)
    iks_out = np.stack([r.iks(10, x) for x in iks_in])
    ksk_rows = np.array([0, 1, 2046 * 5 + 17, 1024 * 2 * 1023 - 1], np.uint64)
    ksk_sample = np.stack([o.ksk_row(10, SEED, keys, int(q) // 2046, (int(q) % 2046) // 1023, int(q) % 1023)
                           for q in ksk_rows])

    bits = rng.integers(0, 2, 4)
    pbs_in = np.stack([o.tlwe32((1 << 29) if b else (-(1 << 29)) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x40, i)
                       for i, b in enumerate(bits)])
    tv = np.full(N1, 1 << 29, np.uint32)
    pbs_out = np.stack([r.pbs01(x, tv) for x in pbs_in])

    np.savez_compressed(
        os.path.join(HERE, "tfhepp_lvl1.npz"),
        seed=np.uint64(SEED), fft_in=fft_in, fft_out=fft_out, fft_back=fft_back,
        dec0=dec[0], dec1=dec[1], dec2=dec[2], iks_in=iks_in, iks_out=iks_out,
        ksk_rows=ksk_rows, ksk_sample=ksk_sample, bk_sample=bk[3, 4, 1, :8].copy(),
        pbs_in=pbs_in, pbs_bit=bits.astype(np.uint8), pbs_out=pbs_out)
    r.close()
    print("wrote", os.path.join(HERE, "tfhepp_lvl1.npz"))
    arcedb(o, s1)


# ArcEDB single-digit comparisons (src/ARCEDB/comparison/comparable.cpp
# 506-523, 652-666, 623-633 and the equal term 537-538), run with the
# reference's TFHEpp steps on encryptions the oracle makes deterministically
# (comparable.h:169-179 and 228-274): inputs are stored as (x, y) and
# regenerated, outputs as the reference computed them.
ARC_OPS = ("gt", "lt", "eq", "equal_term")
ARC_PAIRS = ((0, 0), (0, 1), (1, 0), (700, 699), (1023, 0), (5, 900))


def arcedb(o, s1):
    r = RefTFHEpp()
    out = np.zeros((len(ARC_PAIRS), len(ARC_OPS), N1 + 1), np.uint32)
    for i, (x, y) in enumerate(ARC_PAIRS):
        trl = o.arc_trlwe(x, s1, SEED, 0xA5, i)
        gfft = o.trgsw32_fft(o.arc_trgsw(y, s1, SEED, 0xA6, i))
        for k, op in enumerate(ARC_OPS):
            out[i, k] = r.arc_digit(op, trl, gfft)
    r.close()
    np.savez_compressed(os.path.join(HERE, "arcedb_lvl1.npz"), seed=np.uint64(SEED),
                        pairs=np.array(ARC_PAIRS, np.uint32), out=out)
    print("wrote", os.path.join(HERE, "arcedb_lvl1.npz"))


if __name__ == "__main__":
    main()
