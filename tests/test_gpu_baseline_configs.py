"""GPU results against the FP64 oracle on the benchmark configurations at
their stated sizes, through the C ABI.

- config 1 in full: Doppler, 1e6 lines (2e4 states, J 0-40, nu0 100-10000),
  T = 1500 K, 18 amu, 99,001 bins at 0.1 cm^-1, cutoff 25, Q(T) from the
  device reduction (gexs_partition) within 1e-13 of the oracle's sum;
  FP64 and FP32 forms.
- config 2, a sub-band of the 1e8-line list itself (2e5 states, J 0-80,
  nu0 100-30000, generated on the device with the benchmark's seeds): the
  1e6 lines around its median nu0 on the bins of the 0.01 cm^-1 grid they
  reach, Voigt at 1500 K and 1 bar, FP32 and FP64 forms.
- config 3, eight of the 64 (T, P) pairs over the config-1 list, covering
  T = 100 and 3000 K, P = 1e-5 and 100 bar and all three resolutions (0.1,
  0.01, 0.005 cm^-1 over 100-30000), run as one batch replayed from a CUDA
  graph, each pair against the oracle.
- config 4, a sub-band of the 5e8-line list (1e6 states, J 0-120, nu0
  10-20000): the 1e5 lines around 5000 cm^-1 at 2500 K and P = 1e-3, 1 and
  100 bar, Humlicek and Gauss-Hermite 16 / 32 in the FP32 form (the oracle
  evaluates the same quadrature in FP64).

Tolerances (tests/helpers.py): FP64 form per bin 1e-10 relative (floor
1e-290 for the stable erf form near FP64 underflow); FP32 form 1e-4
relative on bins above 1e-6 of the peak and 1e-6 on the band integral.
"""
import os

import numpy as np
import pytest
import torch

from gexs_b200 import synth, _capi as capi
from gexs_b200.engine import Job, LineList
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu

NTH = len(os.sched_getaffinity(0))
DEV = "cuda"


def _oracle(job, lines):
    return po.cross_section(H.host_job(job.c, lines), nthreads=NTH)


def _check(job, lines, ref=None, what=""):
    got = job.out.cpu().numpy()
    if ref is None:
        ref = _oracle(job, lines)
    s0, s1 = job.c.start_idx, job.c.start_idx + job.c.n_points
    got, ref = got[s0:s1], ref[s0:s1]
    assert np.max(ref) > 0, what
    if job.c.precision == capi.FP64:
        floor = 1e-290 if job.c.profile in (capi.DOPPLER, capi.GAUSSIAN) else 0.0
        worst, nbad = H.fp64_mismatch(got, ref, floor)
        assert nbad == 0, "%s FP64: worst %.3g of tolerance" % (what, worst)
    else:
        rel, band = H.fp32_errors(got, ref)
        assert rel <= H.FP32_REL and band <= H.FP32_BAND, "%s FP32: rel %.3g band %.3g" % (
            what, rel, band)


def _q(ctx, st, temps):
    return ctx.partition(torch.as_tensor(st.energy, device=DEV),
                         torch.as_tensor(st.g, dtype=torch.int32, device=DEV), temps)


@pytest.fixture(scope="module")
def cfg1():
    st = synth.make_states(20000, 40, 1001)
    L = synth.make_lines(st, 1000000, 100.0, 10000.0, 2001, broadening_seed=3001)
    return st, L


def test_config1_doppler_full_size(gpu_ctx, cfg1):
    st, L = cfg1
    q = float(_q(gpu_ctx, st, [1500.0])[0])
    qo = po.partition(st.energy, st.g, 1500.0)
    assert abs(q - qo) <= 1e-13 * qo
    dev = LineList.from_dict(L)
    G = 99001
    for prec in (capi.FP64, capi.FP32):
        j = Job(dev, torch.zeros(G, dtype=torch.float64, device=DEV), convention=capi.CONV_PHYSICAL,
                profile=capi.DOPPLER, temperature=1500.0, pressure=1.0, partition=q, mass=18.0,
                nu_start=100.0, dnu=0.1, grid_points=G, precision=prec, cutoff=25.0)
        assert gpu_ctx.count_evals([j])[0] == po.count_evals(H.host_job(j.c, L)) > 4.9e8
        gpu_ctx.run([j])
        gpu_ctx.check()
        _check(j, L, what="config 1")


def test_config2_subband_of_the_1e8_line_list(gpu_ctx):
    st = synth.make_states(200000, 80, 1002)
    Ld = synth.make_lines_torch(st, 100_000_000, 100.0, 30000.0, 2002, broadening_seed=3002,
                                device=DEV)
    n = Ld["nu"].shape[0]
    a = n // 2 - 500_000
    S = {k: np.ascontiguousarray(v[a:a + 1_000_000].cpu().numpy()) for k, v in Ld.items()}
    del Ld
    torch.cuda.empty_cache()
    q = float(_q(gpu_ctx, st, [1500.0])[0])
    G = 2990001
    j0 = max(0, int(np.floor((S["nu"][0] - 25.0 - 100.0) / 0.01)) - 2)
    j1 = min(G, int(np.ceil((S["nu"][-1] + 25.0 - 100.0) / 0.01)) + 3)
    dev = LineList.from_dict(S)
    for prec in (capi.FP64, capi.FP32):
        j = Job(dev, torch.zeros(G, dtype=torch.float64, device=DEV), convention=capi.CONV_PHYSICAL,
                profile=capi.VOIGT, temperature=1500.0, pressure=1.0, partition=q, mass=18.0,
                nu_start=100.0, dnu=0.01, grid_points=G, precision=prec, cutoff=25.0,
                start_idx=j0, n_points=j1 - j0)
        gpu_ctx.run([j])
        gpu_ctx.check()
        _check(j, S, what="config 2 sub-band")


# (T index, P index, resolution) of the 8 x 8 grid T = logspace(100, 3000),
# P = logspace(1e-5, 100): both T ends, both P ends, all three resolutions
CFG3_PAIRS = [(0, 0, 0.1), (0, 7, 0.01), (7, 0, 0.005), (7, 7, 0.1), (3, 3, 0.01),
              (4, 5, 0.005), (0, 4, 0.1), (7, 2, 0.01)]


def test_config3_pairs_in_one_graph_replayed_batch(gpu_ctx, cfg1):
    st, L = cfg1
    temps = np.logspace(np.log10(100.0), np.log10(3000.0), 8)
    press = np.logspace(-5.0, 2.0, 8)
    qs = _q(gpu_ctx, st, [temps[ti] for ti, _, _ in CFG3_PAIRS])
    dev = LineList.from_dict(L)
    jobs = []
    for (ti, pi, d), q in zip(CFG3_PAIRS, qs):
        G = int(round((30000.0 - 100.0) / d)) + 1
        jobs.append(Job(dev, torch.zeros(G, dtype=torch.float64, device=DEV),
                        convention=capi.CONV_PHYSICAL, profile=capi.VOIGT,
                        temperature=float(temps[ti]), pressure=float(press[pi]),
                        partition=float(q), mass=18.0, nu_start=100.0, dnu=d, grid_points=G,
                        precision=capi.FP32, cutoff=25.0))
    b = gpu_ctx.batch(jobs)
    s = torch.cuda.Stream()
    b.capture(s)
    b.replay(s)
    s.synchronize()
    gpu_ctx.check(s)
    b.close()
    for (ti, pi, d), j in zip(CFG3_PAIRS, jobs):
        _check(j, L, what="config 3 pair T=%g P=%g dnu=%g" % (temps[ti], press[pi], d))


@pytest.fixture(scope="module")
def cfg4():
    st = synth.make_states(1000000, 120, 1004)
    Ld = synth.make_lines_torch(st, 500_000_000, 10.0, 20000.0, 2004, broadening_seed=3004,
                                device=DEV)
    a = int(torch.searchsorted(Ld["nu"], torch.tensor(5000.0, dtype=torch.float64, device=DEV)))
    S = {k: np.ascontiguousarray(v[a - 50_000:a + 50_000].cpu().numpy()) for k, v in Ld.items()}
    del Ld
    torch.cuda.empty_cache()
    return st, S


@pytest.mark.parametrize("P", [1e-3, 1.0, 100.0])
def test_config4_subband_quadrature_and_humlicek(gpu_ctx, cfg4, P):
    st, S = cfg4
    T = 2500.0
    q = float(_q(gpu_ctx, st, [T])[0])
    G = 1999001
    j0 = max(0, int(np.floor((S["nu"][0] - 25.0 - 10.0) / 0.01)) - 2)
    j1 = min(G, int(np.ceil((S["nu"][-1] + 25.0 - 10.0) / 0.01)) + 3)
    dev = LineList.from_dict(S)
    for prof, nodes in ((capi.VOIGT, 16), (capi.VOIGT_QUAD, 16), (capi.VOIGT_QUAD, 32)):
        j = Job(dev, torch.zeros(G, dtype=torch.float64, device=DEV), convention=capi.CONV_PHYSICAL,
                profile=prof, temperature=T, pressure=P, partition=q, mass=18.0, nu_start=10.0,
                dnu=0.01, grid_points=G, precision=capi.FP32, cutoff=25.0, start_idx=j0,
                n_points=j1 - j0, quad_nodes=nodes)
        gpu_ctx.run([j])
        gpu_ctx.check()
        _check(j, S, what="config 4 P=%g %s" % (P, "GH%d" % nodes if prof == capi.VOIGT_QUAD
                                                 else "Humlicek"))
