"""Shared helpers of the test-suite: job construction on device and host,
and the parity checks with their stated tolerances."""
import ctypes as C

import numpy as np

from gexs_b200 import _capi as capi
from gexs_b200.engine import Job, LineList, job_init

# FP64 form vs the FP64 oracle: per-bin relative tolerance
FP64_REL = 1e-10
# FP32-profile form: per-bin relative tolerance on bins above 1e-6 of peak,
# and integrated band intensity
FP32_REL = 1e-4
FP32_FLOOR = 1e-6
FP32_BAND = 1e-6


def host_job(cjob, lines):
    j = capi.GexsJob.from_buffer_copy(cjob)
    def p(a):
        return None if a is None else a.ctypes.data_as(C.c_void_p)
    j.lines = capi.GexsLines(p(lines["nu"]), p(lines["elow"]), p(lines["aif"]), p(lines["gns"]),
                             p(lines.get("gamma")), p(lines.get("n")), len(lines["nu"]))
    j.out = None
    return j


def oracle_of(job, lines, out=None):
    from oracle import pyoracle as po
    hj = host_job(job.c if isinstance(job, Job) else job, lines)
    return po.cross_section(hj, out=out)


def fp64_mismatch(gpu, ref, abs_floor=0.0):
    """max over bins of |gpu-ref| / (FP64_REL*|ref| + abs_floor) (<= 1 passes)."""
    d = np.abs(gpu - ref)
    lim = FP64_REL * np.abs(ref) + abs_floor
    bad = d > lim
    worst = float(np.max(d / np.maximum(lim, 1e-320))) if len(d) else 0.0
    return worst, int(bad.sum())


def fp32_errors(gpu, ref):
    """(max rel error on bins > FP32_FLOOR*peak, band-integral rel error)."""
    peak = float(np.max(np.abs(ref))) if len(ref) else 0.0
    if peak == 0.0:
        return float(np.max(np.abs(gpu))) if len(gpu) else 0.0, 0.0
    m = np.abs(ref) > FP32_FLOOR * peak
    rel = float(np.max(np.abs(gpu[m] - ref[m]) / np.abs(ref[m]))) if m.any() else 0.0
    band = abs(float(np.sum(gpu)) - float(np.sum(ref))) / abs(float(np.sum(ref)))
    return rel, band
