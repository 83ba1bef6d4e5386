"""Cross-section output (gexs_write_sigma): the text form is byte for byte
the reference's OutputProfile text (Profiles/BaseProfile.cpp:289-292),
checked against printf-equivalent formatting of the same values; the binary
form round-trips.  Host arrays, so it runs on the CPU."""
import ctypes as C
import os

import numpy as np

from gexs_b200 import _capi as capi
from gexs_b200._capi import lib


def _sigma(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    s = 10.0 ** rng.uniform(-30, -18, n)
    s[::17] = 0.0
    return s


def _ref_text(index, T, P, nu0, dnu, s):
    lines = ["-------T=%12.6f K--------P=%12.6f atm---------\n\n" % (T, P)]
    lines += ["[%i] %12.6f %13.8E\n" % (index, nu0 + float(j) * dnu, v) for j, v in enumerate(s)]
    lines.append("\n")
    return "".join(lines).encode()


def test_text_is_the_reference_format(tmp_path):
    path = os.path.join(str(tmp_path), "x.txt")
    want = b""
    for idx, (T, P, n) in enumerate([(1500.0, 0.986923, 100003), (296.0, 1e-3, 7), (3000.5, 10.0, 0)]):
        s = _sigma(n, idx)
        st = lib().gexs_write_sigma(path.encode(), capi.OUT_TEXT, 1 if idx else 0, idx, T, P,
                                    100.0, 0.01, n, s.ctypes.data_as(C.c_void_p) if n else None, 4)
        assert st == capi.GEXS_OK
        want += _ref_text(idx, T, P, 100.0, 0.01, s)
    got = open(path, "rb").read()
    assert got == want


def test_binary_round_trip(tmp_path):
    path = os.path.join(str(tmp_path), "x.bin")
    s = _sigma(12345, 3)
    assert lib().gexs_write_sigma(path.encode(), capi.OUT_BINARY, 0, 2, 900.0, 1.5, 50.0, 0.005,
                                  len(s), s.ctypes.data_as(C.c_void_p), 0) == capi.GEXS_OK
    raw = open(path, "rb").read()
    assert raw[:8] == b"GEXSSIG1"
    n = np.frombuffer(raw[8:16], np.int64)[0]
    nu0, dnu, T, P = np.frombuffer(raw[16:48], np.float64)
    idx = np.frombuffer(raw[48:52], np.int32)[0]
    assert (n, nu0, dnu, T, P, idx) == (12345, 50.0, 0.005, 900.0, 1.5, 2)
    back = np.frombuffer(raw[64:], np.float64)
    assert np.array_equal(back, s)


def test_rejects_bad_arguments(tmp_path):
    assert lib().gexs_write_sigma(b"/nonexistent-dir/x", capi.OUT_TEXT, 0, 0, 1.0, 1.0, 0.0, 1.0,
                                  0, None, 1) == capi.GEXS_ERR_INVALID
    assert lib().gexs_write_sigma(os.path.join(str(tmp_path), "y").encode(), 7, 0, 0, 1.0, 1.0,
                                  0.0, 1.0, 0, None, 1) == capi.GEXS_ERR_INVALID
