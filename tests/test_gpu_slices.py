"""Line slices: a tile whose line range holds more than 16384 lines (8192 for
the FP32 Voigt core kernel) is cut into work items whose partial rows the
last slice to finish adds in slice order.  A dense band, 4e5 lines within
20 cm^-1 and a 25 cm^-1 cutoff, puts every line in every tile, so each tile
is split into ~25 slices (region I, FP64 tile kernel, erf tile kernel) and
~13 core slices.  Checked against the FP64 CPU oracle (FP64 form within
1e-10, FP32 forms within the FP32 tolerance) and for bitwise repeatability:
the same job twice, and batched with an unrelated job, give identical bits."""
import numpy as np
import pytest
import torch

from gexs_b200 import Job, LineList, synth, _capi as capi
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu

LO, DNU, G = 970.0, 0.01, 8001


def _setup():
    st = synth.make_states(5000, 40, 4242)
    L = synth.make_lines(st, 400000, 1000.0, 1020.0, 4243, broadening_seed=4244)
    q = po.partition(st.energy, st.g, 1500.0)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"])
    return L, lines, q


def _job(lines, q, profile, precision, T=1500.0):
    out = torch.zeros(G, dtype=torch.float64, device="cuda")
    return Job(lines, out, convention=capi.CONV_PHYSICAL, profile=profile, temperature=T,
               pressure=1.0, partition=q, mass=18.0, nu_start=LO, dnu=DNU, grid_points=G,
               precision=precision, cutoff=25.0)


def test_dense_band_slices_match_oracle(gpu_ctx):
    L, lines, q = _setup()
    for profile in (capi.VOIGT, capi.DOPPLER):
        host = L if profile == capi.VOIGT else {k: v for k, v in L.items() if k not in ("gamma", "n")}
        j64 = _job(lines, q, profile, capi.FP64)
        j32 = _job(lines, q, profile, capi.FP32)
        gpu_ctx.run([j64])
        gpu_ctx.run([j32])
        gpu_ctx.check()
        want = H.oracle_of(j64, host)
        assert np.max(want) > 0
        floor = 1e-14 * np.max(want) if profile == capi.DOPPLER else 0.0
        worst, nbad = H.fp64_mismatch(j64.out.cpu().numpy(), want, abs_floor=floor)
        assert nbad == 0, (profile, worst)
        rel, band = H.fp32_errors(j32.out.cpu().numpy(), want)
        assert rel <= H.FP32_REL and band <= H.FP32_BAND, (profile, rel, band)


def test_dense_band_slices_are_bitwise_repeatable(gpu_ctx):
    L, lines, q = _setup()
    for precision in (capi.FP32, capi.FP64):
        a = _job(lines, q, capi.VOIGT, precision)
        b = _job(lines, q, capi.VOIGT, precision)
        c = _job(lines, q, capi.VOIGT, precision)
        other = _job(lines, q, capi.VOIGT, precision, T=700.0)
        gpu_ctx.run([a])
        gpu_ctx.run([b])
        gpu_ctx.run([other, c])
        gpu_ctx.check()
        ra, rb, rc = (x.out.cpu().numpy().view(np.int64) for x in (a, b, c))
        assert np.array_equal(ra, rb) and np.array_equal(ra, rc), precision
