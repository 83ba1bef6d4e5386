"""Batched launches: many (T, P) pairs with uneven grids in one persistent
launch, captured into a CUDA graph and replayed; results equal the same
jobs run alone (bitwise: every bin sums its lines in the same order) and
match the FP64 oracle within the FP32 tolerances."""
import numpy as np
import pytest
import torch

from gexs_b200 import _capi as capi
from gexs_b200.engine import Job, LineList
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _pairs(lines, prec, n=12, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    temps = np.logspace(2.0, np.log10(3000.0), 4)
    press = np.logspace(-5.0, 2.0, 3)
    jobs = []
    for i in range(n):
        T, P = temps[i % 4], press[(i // 4) % 3]
        d = float(rng.choice([0.1, 0.02, 0.005]))
        G = int(round(3900.0 / d)) + 1
        jobs.append(Job(lines, torch.zeros(G, dtype=torch.float64, device="cuda"),
                        convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T,
                        pressure=P, partition=1500.0 + 10 * i, mass=18.0, nu_start=100.0,
                        dnu=d, grid_points=G, precision=prec, cutoff=25.0))
    return jobs


def test_batch_graph_replay_equals_alone(gpu_ctx, small_lines):
    lines = LineList.from_dict(small_lines)
    batch_jobs = _pairs(lines, capi.FP32)
    alone = _pairs(lines, capi.FP32)
    for j in alone:
        gpu_ctx.run([j], cfg=(4, 8, 0))
    gpu_ctx.check()
    b = gpu_ctx.batch(batch_jobs, cfg=(4, 8, 0))
    s = torch.cuda.Stream()
    b.capture(s)
    for _ in range(2):
        for j in batch_jobs:
            j.out.zero_()
        torch.cuda.synchronize()
        b.replay(s)
        s.synchronize()
        gpu_ctx.check()
        for a, c in zip(batch_jobs, alone):
            assert torch.equal(a.out, c.out)
    b.close()


def test_batch_mixed_profiles_and_precisions(gpu_ctx, small_lines):
    lines = LineList.from_dict(small_lines)
    jobs = _pairs(lines, capi.FP32, n=4) + _pairs(lines, capi.FP64, n=3, seed=9)
    G = 39001
    jobs.append(Job(lines, torch.zeros(G, dtype=torch.float64, device="cuda"),
                    convention=capi.CONV_PHYSICAL, profile=capi.DOPPLER, temperature=900.0,
                    pressure=1.0, partition=1000.0, mass=18.0, nu_start=100.0, dnu=0.1,
                    grid_points=G, precision=capi.FP32, cutoff=25.0))
    b = gpu_ctx.batch(jobs)
    b.launch()
    gpu_ctx.check()
    for j in jobs:
        got = j.out.cpu().numpy()
        ref = H.oracle_of(j, small_lines)
        if j.c.precision == capi.FP64:
            assert H.fp64_mismatch(got, ref)[1] == 0
        else:
            rel, band = H.fp32_errors(got, ref)
            assert rel <= H.FP32_REL and band <= H.FP32_BAND
    b.close()


def test_batch_fp32_vs_oracle_extremes(gpu_ctx, small_lines):
    lines = LineList.from_dict(small_lines)
    jobs = _pairs(lines, capi.FP32, n=12, seed=11)
    b = gpu_ctx.batch(jobs)
    b.launch()
    gpu_ctx.check()
    for j in jobs:
        rel, band = H.fp32_errors(j.out.cpu().numpy(), H.oracle_of(j, small_lines))
        assert rel <= H.FP32_REL and band <= H.FP32_BAND, (j.c.temperature if hasattr(j.c, "temperature") else None, rel, band)
    b.close()


def test_autotune_returns_a_valid_shape(gpu_ctx, small_lines):
    lines = LineList.from_dict(small_lines)
    jobs = _pairs(lines, capi.FP32, n=3)
    cfg, ms = gpu_ctx.autotune(jobs)
    assert cfg[0] in (2, 4, 8, 16) and cfg[1] in (4, 8) and ms > 0
    # flags: at most the stage length and, for several jobs, the item order
    assert cfg[3] & ~(capi.LAUNCH_LONG_STAGES | capi.LAUNCH_JOB_MAJOR) == 0
    # the tuned launch is the context default now: same bits as tile-major
    a = _pairs(lines, capi.FP32, n=3)
    b = _pairs(lines, capi.FP32, n=3)
    gpu_ctx.run(a)
    gpu_ctx.run(b, cfg=(4, 4, 0, capi.LAUNCH_LONG_STAGES))
    gpu_ctx.check()
    if cfg[:2] == (4, 4) and cfg[3] & capi.LAUNCH_LONG_STAGES:
        for x, y in zip(a, b):
            assert torch.equal(x.out, y.out)
