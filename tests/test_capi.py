"""C ABI surface, checked without a GPU: every function declared in
include/*.h is exported by libgexs_b200.so, the convention presets
reproduce the reference's constants, and bad arguments are rejected
before any CUDA call."""
import ctypes as C
import os
import re

import pytest

from gexs_b200 import _capi as capi
from gexs_b200.engine import job_init

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(gexs_[a-z0-9_]+)\s*\(", txt))
    return names


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(capi.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 30
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    bound = {s[0] for s in capi.SIGNATURES}
    assert _declared() <= bound | {"gexs_probe_fp32_tflops"} | bound


def test_status_strings():
    L = capi.lib()
    for code in (0, -1, -2, -3, -4, -5, -6, -7, -8):
        assert L.gexs_status_string(code)
    assert L.gexs_status_string(-99) == b"unknown status"


def test_reference_cpu_preset():
    j = job_init(capi.CONV_REF_CPU, capi.VOIGT, 1500.0, 2.0, 1000.0, 18.0, 100.0, 0.01, 1000)
    assert j.window_rule == capi.WINDOW_ROUNDED
    assert j.erf_form == capi.ERF_LITERAL
    assert j.cutoff == 50.0                      # min(25 P, 100)
    assert j.s_scale2 == 0.564189584             # ISQRTPI inside S
    assert j.gamma_scale == 1.0                  # no pressure factor
    assert j.s_scale == 1.0 / (8.0 * 3.14159265359 * 2.99792458e10)
    j = job_init(capi.CONV_REF_CPU, capi.VOIGT, 1500.0, 9.0, 1000.0, 18.0, 100.0, 0.01, 1000)
    assert j.cutoff == 100.0
    d = job_init(capi.CONV_REF_CPU, capi.DOPPLER, 1500.0, 1.0, 1000.0, 18.0, 100.0, 0.01, 1000)
    assert d.cutoff == 100.0 and d.out_scale == 1.0 and d.s_scale2 == 1.0


def test_physical_preset():
    import math
    j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, 1500.0, 1.01325, 1000.0, 18.0, 100.0, 0.01, 10,
                 cutoff=25.0)
    assert j.window_rule == capi.WINDOW_INCLUSIVE and j.cutoff == 25.0
    assert abs(j.gamma_scale - 1.0) < 1e-15       # 1.01325 bar = 1 atm
    assert abs(j.out_scale - 1.0 / math.sqrt(math.pi)) < 1e-16
    # 1/e Doppler half width of an 18 amu molecule at 1500 K: ~3.93e-6 per cm^-1
    assert 3.9e-6 < j.dop_coef < 3.96e-6
    d = job_init(capi.CONV_PHYSICAL, capi.DOPPLER, 1500.0, 1.0, 1000.0, 18.0, 100.0, 0.01, 10)
    assert d.out_scale == 0.5 / 0.01


def test_bad_arguments_are_rejected_on_cpu():
    L = capi.lib()
    j = capi.GexsJob()
    assert L.gexs_job_init(C.byref(j), 0, capi.VOIGT, -1.0, 1.0, 1.0, 18.0, 296.0, 1.0, 0.0,
                           -1.0, 100.0, 0.01, 10) == -1
    assert L.gexs_job_init(C.byref(j), 7, capi.VOIGT, 100.0, 1.0, 1.0, 18.0, 296.0, 1.0, 0.0,
                           -1.0, 100.0, 0.01, 10) == -1
    assert L.gexs_run(None, None, 0, None, None) == -1
    assert L.gexs_run_noalloc(None, 0, None, None) == -1
    assert L.gexs_count_evals(None, None, 0, None) == -1
    assert L.gexs_batch_launch(None, None) == -1
    assert L.gexs_manager_execute(None, 1, 1, 0, 1.0, 1.0, 1.0) == -1
    assert L.gexs_server_submit(None, None, None) == -1
    assert L.gexs_manager_create_multi(capi.VOIGT, None, 1, 0, 0, 0, None) == -1
    assert L.gexs_shard_plan(None, 5, 0.0, 1.0, 0, 10, 1.0, 4096, 2, None, None, None) == -1
