"""Packs of pairs in the FP32 Voigt region-I kernel (gexs_launch_cfg.pairs):
jobs that share the grid, the cutoff, the window rule and the line list are
evaluated together per tile, each staged chunk of lines and each line's
window shared by the pairs.  A pair's bins sum its records exactly as
without packs, so results are bitwise those of pairs = 1 - on a sparse list,
on a dense band whose tiles are cut into line slices (partial rows and
tickets per (tile, pair)), with lines derived on load, in a graph-replayed
batch, and for jobs of two grids mixed in one launch (packs form per grid).
Each is also within the FP32 tolerance of the FP64 oracle (1e-4 relative on
bins above 1e-6 of the peak, band integral 1e-6).  Lines per stage (64 or
128) change where the FP32 partial sums fold into the Kahan pairs, so there
only the tolerance applies.
"""
import pytest
import torch

from gexs_b200 import Context, Job, LineList, synth, _capi as capi
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu

TP = [(1500.0, 1.0), (300.0, 1e-3), (2500.0, 30.0), (800.0, 0.2), (1200.0, 5.0), (100.0, 1e-5),
      (2000.0, 0.05)]


def _jobs(lines, q_of, grids, prec=capi.FP32):
    jobs = []
    for i, (T, P) in enumerate(TP):
        nu0, dnu, G = grids[i % len(grids)]
        out = torch.zeros(G, dtype=torch.float64, device="cuda")
        jobs.append(Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT,
                        temperature=T, pressure=P, partition=q_of(T), mass=18.0, nu_start=nu0,
                        dnu=dnu, grid_points=G, precision=prec, cutoff=25.0))
    return jobs


def _run(ctx, lines, q_of, grids, cfg):
    jobs = _jobs(lines, q_of, grids)
    ctx.run(jobs, cfg=cfg)
    ctx.check()
    return jobs


def _same(a, b):
    for x, y in zip(a, b):
        assert torch.equal(x.out, y.out)


def _oracle_ok(jobs, host):
    for j in jobs:
        want = H.oracle_of(j, host)
        rel, band = H.fp32_errors(j.out.cpu().numpy(), want)
        assert rel <= H.FP32_REL and band <= H.FP32_BAND, (j.c.temperature, rel, band)


def test_packs_bitwise_equal_single_pairs(gpu_ctx, small_states, small_lines):
    lines = LineList.from_dict(small_lines)
    q_of = lambda T: po.partition(small_states.energy, small_states.g, T)
    grids = [(100.0, 0.05, 80000), (600.0, 0.02, 60001)]
    ref = _run(gpu_ctx, lines, q_of, grids, (4, 4, 0, 0, 0, 1))
    for pp in (2, 4):
        _same(_run(gpu_ctx, lines, q_of, grids, (4, 4, 0, 0, 0, pp)), ref)
        _same(_run(gpu_ctx, lines, q_of, grids, (8, 4, 0, 0, 0, pp)),
              _run(gpu_ctx, lines, q_of, grids, (8, 4, 0, 0, 0, 1)))
    # lines derived on load (no prep arrays) with packs
    on_load = _run(gpu_ctx, lines, q_of, grids, (4, 4, 0, capi.LAUNCH_DERIVE_ON_LOAD, 0, 1))
    _same(_run(gpu_ctx, lines, q_of, grids, (4, 4, 0, capi.LAUNCH_DERIVE_ON_LOAD, 0, 4)), on_load)
    _oracle_ok(ref, small_lines)


def test_packs_on_sliced_dense_band(gpu_ctx):
    st = synth.make_states(5000, 40, 4242)
    L = synth.make_lines(st, 200000, 1000.0, 1020.0, 4243, broadening_seed=4244)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"])
    q_of = lambda T: po.partition(st.energy, st.g, T)
    grids = [(970.0, 0.01, 8001)]
    ref = _run(gpu_ctx, lines, q_of, grids, (4, 4, 0, 0, 0, 1))
    for pp in (2, 4):
        _same(_run(gpu_ctx, lines, q_of, grids, (4, 4, 0, 0, 0, pp)), ref)
    _oracle_ok(ref[:3], L)


def test_packs_in_a_graph_replayed_batch(gpu_ctx, small_states, small_lines):
    lines = LineList.from_dict(small_lines)
    q_of = lambda T: po.partition(small_states.energy, small_states.g, T)
    grids = [(100.0, 0.05, 80000)]
    ref = _run(gpu_ctx, lines, q_of, grids, (4, 4, 0, 0, 0, 1))
    jobs = _jobs(lines, q_of, grids)
    b = gpu_ctx.batch(jobs, (4, 4, 0, 0, 0, 4))
    s = torch.cuda.Stream()
    b.capture(s)
    for _ in range(2):
        b.replay(s)
    s.synchronize()
    gpu_ctx.check(s)
    b.close()
    _same(jobs, ref)


def test_lines_per_stage(gpu_ctx, small_states, small_lines):
    lines = LineList.from_dict(small_lines)
    q_of = lambda T: po.partition(small_states.energy, small_states.g, T)
    for pp in (1, 4):
        jobs = _run(gpu_ctx, lines, q_of, [(100.0, 0.05, 80000)], (4, 4, 0, 0, 0, pp, 64))
        _oracle_ok(jobs, small_lines)


def test_autotune_reports_a_pack_shape(small_states, small_lines):
    ctx = Context(0)           # tuning sets a context's default shape
    lines = LineList.from_dict(small_lines)
    q_of = lambda T: po.partition(small_states.energy, small_states.g, T)
    jobs = _jobs(lines, q_of, [(100.0, 0.05, 80000)])
    cfg, ms = ctx.autotune(jobs)
    assert ms > 0 and cfg[5] in (0, 1, 2, 4) and cfg[6] in (0, 64, 128)
    ctx.run(jobs, cfg=cfg)
    ctx.check()
    _oracle_ok(jobs[:2], small_lines)
    ctx.close()
