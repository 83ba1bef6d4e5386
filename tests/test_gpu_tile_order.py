"""Work-item order of a launch with several jobs.  By default the items go
tile-major (tile t of every job that has one, then tile t + 1), so the
(T, P) pairs of a batch over one line list read a tile's lines while they
sit in L2; GEXS_LAUNCH_JOB_MAJOR restores job-major order.  A tile's sums do
not depend on which CTA runs it or when, so both orders, and every job run
alone, must give the same bits.  The jobs have uneven tile counts (grid
sub-ranges, a one-point job, different spacings), so the order tables have
several segments, and the dense band splits every tile into line slices."""
import numpy as np
import pytest
import torch

from gexs_b200 import Job, LineList, synth, _capi as capi
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu

LO = 970.0


def _dense():
    st = synth.make_states(5000, 40, 4242)
    L = synth.make_lines(st, 400000, 1000.0, 1020.0, 4243, broadening_seed=4244)
    q = po.partition(st.energy, st.g, 1500.0)
    return L, LineList.from_dict(L), q


def _jobs(lines, q, profile, precision):
    """five (T, P) pairs, tile counts uneven: grid spacing, sub-range and a
    one-point job"""
    spec = [  # (T, P, dnu, start_idx, n_points)
        (1500.0, 1.0, 0.01, 0, None),
        (300.0, 1e-3, 0.01, 3500, 1500),
        (2500.0, 10.0, 0.02, 0, None),
        (800.0, 0.1, 0.01, 4321, 1),
        (1200.0, 3.0, 0.01, 3000, 5001),
    ]
    jobs = []
    for T, P, d, s0, n in spec:
        G = int(round(80.0 / d)) + 1
        jobs.append(Job(lines, torch.zeros(G, dtype=torch.float64, device="cuda"),
                        convention=capi.CONV_PHYSICAL, profile=profile, temperature=T,
                        pressure=P, partition=q, mass=18.0, nu_start=LO, dnu=d, grid_points=G,
                        precision=precision, cutoff=25.0, start_idx=s0, n_points=n))
    return jobs


CASES = [  # (profile, precision, launch shape and flags)
    (capi.VOIGT, capi.FP32, (4, 4, 0, capi.LAUNCH_LONG_STAGES)),
    (capi.VOIGT, capi.FP32, (2, 8, 0, 0)),
    (capi.VOIGT, capi.FP64, (4, 8, 0, 0)),
    (capi.DOPPLER, capi.FP32, (4, 4, 0, 0)),
]


@pytest.mark.parametrize("profile,precision,cfg", CASES)
def test_tile_major_equals_job_major_and_alone(gpu_ctx, profile, precision, cfg):
    L, lines, q = _dense()
    tile_major = _jobs(lines, q, profile, precision)
    job_major = _jobs(lines, q, profile, precision)
    alone = _jobs(lines, q, profile, precision)
    gpu_ctx.run(tile_major, cfg=cfg)
    gpu_ctx.run(job_major, cfg=cfg[:3] + (cfg[3] | capi.LAUNCH_JOB_MAJOR,))
    for j in alone:
        gpu_ctx.run([j], cfg=cfg)
    gpu_ctx.check()
    for a, b, c in zip(tile_major, job_major, alone):
        assert float(a.out.abs().max()) > 0 or a.c.n_points == 1
        assert torch.equal(a.out, b.out)
        assert torch.equal(a.out, c.out)


def test_tile_major_batch_matches_oracle(gpu_ctx, small_lines):
    """the graph-captured batch (tile-major by default) on a sparse list
    against the FP64 oracle"""
    lines = LineList.from_dict(small_lines)
    jobs = []
    for i, (T, P, d) in enumerate([(300.0, 1e-3, 0.1), (1500.0, 1.0, 0.02), (2800.0, 50.0, 0.05)]):
        G = int(round(3900.0 / d)) + 1
        jobs.append(Job(lines, torch.zeros(G, dtype=torch.float64, device="cuda"),
                        convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T,
                        pressure=P, partition=1500.0 + 10 * i, mass=18.0, nu_start=100.0,
                        dnu=d, grid_points=G, precision=capi.FP32, cutoff=25.0))
    b = gpu_ctx.batch(jobs)
    s = torch.cuda.Stream()
    b.capture(s)
    b.replay(s)
    s.synchronize()
    gpu_ctx.check()
    for j in jobs:
        rel, band = H.fp32_errors(j.out.cpu().numpy(), H.oracle_of(j, small_lines))
        assert rel <= H.FP32_REL and band <= H.FP32_BAND
    b.close()
