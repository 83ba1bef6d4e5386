"""gexs_write_sigma from a device array gives the same bytes as from the
host copy of it (the device path copies out, then formats)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from gexs_b200 import _capi as capi
from gexs_b200._capi import lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", [capi.OUT_TEXT, capi.OUT_BINARY])
def test_device_and_host_sigma_write_the_same_bytes(tmp_path, fmt):
    rng = np.random.Generator(np.random.PCG64(5))
    s = 10.0 ** rng.uniform(-28, -19, 300001)
    d = torch.as_tensor(s, device="cuda")
    ph, pd = os.path.join(str(tmp_path), "h"), os.path.join(str(tmp_path), "d")
    assert lib().gexs_write_sigma(ph.encode(), fmt, 0, 1, 1200.0, 1.0, 100.0, 0.01, len(s),
                                  s.ctypes.data_as(C.c_void_p), 0) == capi.GEXS_OK
    assert lib().gexs_write_sigma(pd.encode(), fmt, 0, 1, 1200.0, 1.0, 100.0, 0.01, len(s),
                                  C.c_void_p(d.data_ptr()), 0) == capi.GEXS_OK
    assert open(ph, "rb").read() == open(pd, "rb").read()
