"""The bounded waits of the FP32 Voigt pipeline (voigt_ws_kernel): with
one try_wait attempt per wait (gexs_launch_cfg.wait_spins = 1) a hand-over
wait runs out; the kernel flags GEXS_KERR_PIPELINE and returns instead of
hanging, gexs_ctx_check reports GEXS_ERR_KERNEL and clears the word, and the
context then runs the same job correctly (FP32 tolerance against the FP64
oracle: 1e-4 relative on bins above 1e-6 of the peak, band 1e-6)."""
import pytest
import torch

from gexs_b200 import _capi as capi
from gexs_b200.engine import Job, LineList
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _job(lines):
    out = torch.zeros(30000, dtype=torch.float64, device="cuda")
    return Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT,
               temperature=1500.0, pressure=0.5, partition=2000.0, mass=18.0, nu_start=150.0,
               dnu=0.1, grid_points=30000, precision=capi.FP32, cutoff=25.0)


def test_wait_limit_runs_out_then_context_recovers(gpu_ctx, small_lines):
    lines = LineList.from_dict(small_lines)
    gpu_ctx.check()                                  # start from a clear word
    j = _job(lines)
    gpu_ctx.run([j], cfg=(4, 4, 0, 0, 1))
    with pytest.raises(capi.GexsError) as ei:
        gpu_ctx.check()
    assert ei.value.status == capi.GEXS_ERR_KERNEL
    gpu_ctx.check()                                  # the check cleared it
    j2 = _job(lines)
    gpu_ctx.run([j2])
    gpu_ctx.check()
    ref = H.oracle_of(j2, small_lines)
    rel, band = H.fp32_errors(j2.out.cpu().numpy(), ref)
    assert rel <= H.FP32_REL and band <= H.FP32_BAND, (rel, band)
