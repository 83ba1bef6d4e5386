"""The reference's own GPU path (GpuManager, Managers/Accel/GPU/GPUManager.cpp,
with the v2 Voigt kernel of compute/CUDA/cross_kernal_v2.cu:403-457 and its
FP32 Humlicek humlickf :52-84), compiled from its sources for sm_100a as
oracle/_ref/gexsref_gpu, against our reference-GPU convention
(GEXS_CONV_REF_GPU: 1/e Doppler width, gamma (T_ref/T)^n P ref_press,
inclusive 100 cm^-1 window) on the same lines and bins.  The reference
evaluates W4 in FP32, so the bound is FP32-sized: every bin above 1e-6 of
the peak within 3e-6 relative, the integral within 1e-6."""
import numpy as np
import pytest
import torch

from gexs_b200 import Context, Job, LineList, synth, _capi as capi
from oracle import pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.ref_gpu_available(),
                                 reason="reference GPU harness not built (oracle/_ref)")]

REL, BAND = 3e-6, 1e-6


@pytest.mark.parametrize("T,P", [(1500.0, 1.0), (300.0, 0.05)])
def test_reference_gpu_kernel_matches_ref_gpu_convention(T, P):
    st = synth.make_states(20000, 40, 11)
    L = synth.make_lines(st, 200000, 1000.0, 1400.0, 12, broadening_seed=13)
    q = po.partition(st.energy, st.g, T)
    lo, dnu, nb = 900.0, 0.01, 60001
    sig, ms = po.ref_gpu_voigt(L, lo, dnu, nb, T, P, q, 18.0, 296.0, 1.0, 0.0, reps=1)
    assert len(ms) == 1 and sig.shape == (nb,)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"])
    ctx = Context(0)
    for prec in (capi.FP64, capi.FP32):
        out = torch.zeros(nb, dtype=torch.float64, device="cuda")
        j = Job(lines, out, convention=capi.CONV_REF_GPU, profile=capi.VOIGT, temperature=T,
                pressure=P, partition=q, mass=18.0, nu_start=lo, dnu=dnu, grid_points=nb,
                precision=prec, ref_temp=296.0, ref_press=1.0)
        ctx.run([j])
        ctx.check()
        o = out.cpu().numpy()
        m = o > 1e-6 * o.max()
        rel = np.abs(sig[m] - o[m]) / o[m]
        assert rel.max() <= REL, (prec, float(rel.max()))
        assert abs(sig.sum() - o.sum()) <= BAND * o.sum()
