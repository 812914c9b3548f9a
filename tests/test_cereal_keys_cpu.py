"""Key material I/O: the reference's cereal key archives
(src/HEDB/utils/serialize.cpp:7-60 -- cereal::PortableBinaryOutputArchive of
TFHEpp EvalKey::serialize_<key>, thirdparty/TFHEpp/include/cloudkey.hpp:
149-228), checked without a GPU.

Archives are written by the reference's own TFHEpp (oracle/_ref) from the
deterministic key set; the engine's host-only locator
(cufhedb_cereal_key_payload) must find in them exactly the bytes of the key
TFHEpp holds in memory, and refuse files that do not hold the key asked for.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import SEED

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from cufhedb_b200 import _lib
    return _lib.load()


def _payload(lib, path, kind):
    off, n = C.c_uint64(0), C.c_uint64(0)
    rc = lib.cufhedb_cereal_key_payload(path.encode(), kind, C.byref(off), C.byref(n))
    return rc, off.value, n.value


def test_bkfft01_archive_payload_is_tfhepp_key(lib, ref_keyed, tmp_path):
    path = str(tmp_path / "bkfftlvl01.key")
    ref_keyed.save_cereal("bkfft01", path)
    rc, off, n = _payload(lib, path, 1)
    assert rc == 0
    want = ref_keyed.bkfft01()
    assert n == want.nbytes and off + n == os.path.getsize(path)
    got = np.fromfile(path, dtype=np.float64, offset=off, count=want.size).reshape(want.shape)
    assert np.array_equal(got, want)
    # the same file is not a lvl02 key nor a key-switching key
    for kind in (2, 10, 20, 21):
        assert _payload(lib, path, kind)[0] == 1


def test_ksk21_archive_payload_is_tfhepp_key(lib, ref_keyed, oracle, keys, tmp_path):
    ptr, view = ref_keyed.ksk_view(21)
    oracle.ksk_full_into(21, SEED, keys, ptr)
    path = str(tmp_path / "iksklvl21.key")
    ref_keyed.save_cereal("ksk21", path)
    rc, off, n = _payload(lib, path, 21)
    assert rc == 0 and n == view.nbytes
    rows = np.random.default_rng(3).integers(0, view.shape[0], 64)
    with open(path, "rb") as f:
        for r in rows:
            f.seek(off + int(r) * view.shape[1] * 4)
            assert np.array_equal(np.frombuffer(f.read(view.shape[1] * 4), np.uint32), view[r])
    os.unlink(path)


def test_damaged_archives_are_refused(lib, ref_keyed, tmp_path):
    path = str(tmp_path / "bk.key")
    ref_keyed.save_cereal("bkfft01", path)
    raw = open(path, "rb").read()
    _, off, n = _payload(lib, path, 1)
    big_endian = bytes([0]) + raw[1:]
    empty_ptr = raw[:off - 1] + bytes([0]) + raw[off:]
    for bad in (big_endian, empty_ptr, raw[:len(raw) // 2]):
        p = str(tmp_path / "bad.key")
        open(p, "wb").write(bad)
        assert _payload(lib, p, 1)[0] == 1
    assert _payload(lib, str(tmp_path / "missing.key"), 1)[0] == 1
