"""gexs_run_noalloc: the launch path for callers that must not allocate
device memory while they run (a plug-in whose host program owns all GPU
memory, or a loop where a device allocation could stall or fail).  It keeps
its launch tables and work counter in a fixed array in the library instead
of memory from cudaMallocAsync.

Checked through the C ABI against gexs_run on two calls in a row, with the
tolerances of the other GPU tests (FP64: 1e-10 relative per bin; FP32:
1e-4 relative on bins above 1e-6 of the peak, band 1e-6).  The second call
also shows that the shared work counter starts from zero again.  Around the
calls the device's free memory and torch's allocator stay unchanged, and
gexs_noalloc_status reads a clear error word; a call whose bounded waits
are given one attempt each reports GEXS_ERR_KERNEL there, and the next call
starts from a clear word.  This file sorts last so a stop-at-first-failure
run has run every other test first; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from gexs_b200 import _capi as capi
from gexs_b200.engine import Job, LineList, _job_array
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _jobs(lines, prec, temps, G=30000):
    out = []
    for T in temps:
        out.append(Job(lines, torch.zeros(G, dtype=torch.float64, device="cuda"),
                       convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T,
                       pressure=0.5, partition=2000.0, mass=18.0, nu_start=150.0, dnu=0.1,
                       grid_points=G, precision=prec, cutoff=25.0))
    return out


def _noalloc(jobs, cfg=None):
    arr = _job_array(jobs)
    c = None if cfg is None else C.byref(capi.GexsLaunchCfg(*cfg))
    st = capi.lib().gexs_run_noalloc(arr, len(arr), c, None)
    capi.check(st, "gexs_run_noalloc")


def _status():
    flags = C.c_int(-1)
    st = capi.lib().gexs_noalloc_status(None, C.byref(flags))
    return st, flags.value


def _compare(a, b, prec):
    if prec == capi.FP64:
        worst, nbad = H.fp64_mismatch(a, b)
        assert nbad == 0, "worst %.3g of tolerance" % worst
    else:
        rel, band = H.fp32_errors(a, b)
        assert rel <= H.FP32_REL and band <= H.FP32_BAND, (rel, band)


@pytest.mark.parametrize("prec", [capi.FP32, capi.FP64])
def test_noalloc_matches_run_twice(gpu_ctx, small_lines, prec):
    """Both entry points at their default launch shape (cfg NULL)."""
    lines = LineList.from_dict(small_lines)
    for call, temps in enumerate(([700.0, 1500.0, 2900.0], [300.0, 1200.0])):
        ref_jobs = _jobs(lines, prec, temps)
        na_jobs = _jobs(lines, prec, temps)
        gpu_ctx.run(ref_jobs)
        gpu_ctx.check()
        _noalloc(na_jobs)
        assert _status() == (capi.GEXS_OK, 0)
        for r, n in zip(ref_jobs, na_jobs):
            a, b = n.out.cpu().numpy(), r.out.cpu().numpy()
            assert np.max(b) > 0, "call %d produced an empty reference" % call
            _compare(a, b, prec)


def test_noalloc_allocates_nothing(small_lines):
    lines = LineList.from_dict(small_lines)
    jobs = _jobs(lines, capi.FP32, [900.0, 2100.0])
    _noalloc(jobs)                      # first call: symbol lookup, module load
    assert _status() == (capi.GEXS_OK, 0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(2):
        _noalloc(jobs)
        assert _status() == (capi.GEXS_OK, 0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, "device free memory changed by %d bytes" % (free0 - free1)
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_reports_a_wait_that_ran_out(small_lines):
    """One try_wait attempt per bounded wait of the FP32 Voigt pipeline: a
    wait runs out, the kernel flags it and returns; the next call with the
    default limit starts from a clear word and gives the right result."""
    lines = LineList.from_dict(small_lines)
    bad = _jobs(lines, capi.FP32, [1500.0])
    _noalloc(bad, cfg=(4, 4, 0, 0, 1))
    st, flags = _status()
    assert st == capi.GEXS_ERR_KERNEL and flags & capi.KERR_PIPELINE, (st, flags)
    good = _jobs(lines, capi.FP32, [1500.0])
    ref = _jobs(lines, capi.FP32, [1500.0])
    _noalloc(good)
    assert _status() == (capi.GEXS_OK, 0)
    _noalloc(ref, cfg=(4, 4, 0, 0, 0))
    assert _status() == (capi.GEXS_OK, 0)
    assert torch.equal(good[0].out, ref[0].out)
    assert float(good[0].out.max()) > 0


def test_noalloc_rejects_oversize_and_mixed_calls(small_lines):
    lines = LineList.from_dict(small_lines)
    many = _jobs(lines, capi.FP32, [1000.0] * (capi.NOALLOC_MAX_JOBS + 1), G=100)
    arr = _job_array(many)
    assert capi.lib().gexs_run_noalloc(arr, len(arr), None, None) == -1
    assert b"njobs" in capi.lib().gexs_last_error()
    mixed = _jobs(lines, capi.FP32, [1000.0], G=100) + _jobs(lines, capi.FP64, [1000.0], G=100)
    arr = _job_array(mixed)
    assert capi.lib().gexs_run_noalloc(arr, len(arr), None, None) == -1
