"""GPU kernels vs the FP64 oracle, through the C ABI (gexs_run).

Tolerances (stated in tests/helpers.py):
  FP64 form: per bin |gpu - oracle| <= 1e-10 |oracle| (+ a floor of 1e-290
    for the stable erf form near FP64 underflow, or 1e-14 of the peak for
    the literal erf(xp)-erf(xm) form whose far wing is rounding noise);
  FP32-profile form: per bin relative 1e-4 on bins above 1e-6 of the peak,
    band integral relative 1e-6.
"""
import numpy as np
import pytest
import torch

from gexs_b200 import _capi as capi
from gexs_b200.engine import Job, LineList
from tests import helpers as H

pytestmark = pytest.mark.gpu

PROFILES = [
    ("voigt", capi.VOIGT, 16),
    ("doppler", capi.DOPPLER, 16),
    ("gauss", capi.GAUSSIAN, 16),
    ("gh16", capi.VOIGT_QUAD, 16),
    ("gh32", capi.VOIGT_QUAD, 32),
]


def _make(lines_np, prec, profile, nodes, conv, T=1500.0, P=1.0, G=40000, nu0=100.0, dnu=0.1,
          cutoff=-1.0, start_idx=0, n_points=None, accumulate=0, half_width=0.2,
          out=None, lines_dev=None):
    L = lines_dev if lines_dev is not None else LineList.from_dict(lines_np)
    if out is None:
        out = torch.zeros(G, dtype=torch.float64, device="cuda")
    j = Job(L, out, convention=conv, profile=profile, temperature=T, pressure=P,
            partition=1234.5, mass=18.0, nu_start=nu0, dnu=dnu, grid_points=G,
            precision=prec, half_width=half_width, cutoff=cutoff, start_idx=start_idx,
            n_points=n_points, accumulate=accumulate, quad_nodes=nodes, ref_temp=296.0)
    return j


def _floor(job, ref):
    if job.c.profile in (capi.DOPPLER, capi.GAUSSIAN):
        if job.c.erf_form == capi.ERF_LITERAL:
            return 1e-14 * float(np.max(np.abs(ref)))
        return 1e-290
    return 0.0


def _check(gpu_ctx, job, lines_np, init=None):
    gpu_ctx.run([job])
    gpu_ctx.check()
    got = job.out.cpu().numpy()
    ref = H.oracle_of(job, lines_np, out=None if init is None else init.copy())
    if job.c.precision == capi.FP64:
        worst, nbad = H.fp64_mismatch(got, ref, _floor(job, ref))
        assert nbad == 0, "FP64 mismatch: worst %.3g of tolerance" % worst
    else:
        rel, band = H.fp32_errors(got, ref)
        assert rel <= H.FP32_REL, "FP32 per-bin rel %.3g" % rel
        assert band <= H.FP32_BAND, "FP32 band rel %.3g" % band
    return got, ref


@pytest.mark.parametrize("name,profile,nodes", PROFILES)
@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("conv", [capi.CONV_PHYSICAL, capi.CONV_REF_CPU])
def test_profiles_match_oracle(gpu_ctx, small_lines, name, profile, nodes, prec, conv):
    job = _make(small_lines, prec, profile, nodes, conv)
    got, ref = _check(gpu_ctx, job, small_lines)
    assert np.max(ref) > 0


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_voigt_low_pressure_all_regions(gpu_ctx, small_lines, prec):
    """P = 1e-4 bar: y << 1 so regions III and IV occur near every core."""
    from oracle import pyoracle as po
    job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_PHYSICAL, T=2500.0, P=1e-4,
                dnu=0.002, G=200000, nu0=3000.0)
    hist = po.region_hist(H.host_job(job.c, small_lines))
    assert hist[3] > 0 and hist[2] > 0
    _check(gpu_ctx, job, small_lines)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_voigt_high_pressure(gpu_ctx, small_lines, prec):
    job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_PHYSICAL, T=300.0, P=100.0,
                cutoff=100.0)
    _check(gpu_ctx, job, small_lines)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_reference_gpu_convention(gpu_ctx, small_lines, prec):
    job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_REF_GPU)
    _check(gpu_ctx, job, small_lines)


def test_empty_line_list(gpu_ctx, small_lines):
    empty = {k: v[:0] for k, v in small_lines.items()}
    for prec in (capi.FP64, capi.FP32):
        job = _make(empty, prec, capi.VOIGT, 16, capi.CONV_PHYSICAL, G=5000)
        job.out.fill_(7.0)
        gpu_ctx.run([job]); gpu_ctx.check()
        assert torch.count_nonzero(job.out).item() == 0


def test_lines_outside_grid(gpu_ctx, small_lines):
    for prec in (capi.FP64, capi.FP32):
        job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_PHYSICAL, nu0=20000.0, G=3000)
        gpu_ctx.run([job]); gpu_ctx.check()
        assert torch.count_nonzero(job.out).item() == 0


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_line_exactly_at_cutoff(gpu_ctx, prec):
    """Lines whose distance to a bin equals the cutoff exactly: the
    inclusive rule keeps that bin on both sides."""
    nu0, dnu, cut, G = 1000.0, 0.5, 2.0, 64
    nus = np.array([1002.0 + 2.0, 1010.0 - 2.0, 1016.25, 1020.0], dtype=np.float64)
    lines = {"nu": nus, "elow": np.array([100.0, 200.0, 300.0, 400.0]),
             "aif": np.array([1.0, 2.0, 3.0, 4.0]), "gns": np.array([3, 5, 7, 9], np.int32),
             "gamma": np.array([0.05, 0.06, 0.07, 0.08]), "n": np.array([0.5, 0.6, 0.7, 0.5])}
    for profile in (capi.VOIGT, capi.DOPPLER):
        job = _make(lines, prec, profile, 16, capi.CONV_PHYSICAL, nu0=nu0, dnu=dnu, G=G,
                    cutoff=cut, T=3000.0)
        got, ref = _check(gpu_ctx, job, lines)
        if profile == capi.VOIGT:
            # bin 4 (f = 1002) is exactly cut below the first line
            assert ref[4] > 0 and got[4] > 0 and ref[3] == 0 and got[3] == 0


@pytest.mark.parametrize("G", [1, 37, 1023, 1025, 2049, 4097])
def test_ragged_grids(gpu_ctx, small_lines, G):
    for prec in (capi.FP64, capi.FP32):
        job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_PHYSICAL, nu0=1500.0, dnu=0.01, G=G)
        _check(gpu_ctx, job, small_lines)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_subrange_and_accumulate(gpu_ctx, small_lines, prec):
    G = 40000
    init = np.linspace(1e-20, 2e-20, G)
    out = torch.as_tensor(init.copy(), device="cuda")
    job = _make(small_lines, prec, capi.VOIGT, 16, capi.CONV_REF_CPU, G=G, start_idx=5000,
                n_points=17777, accumulate=1, out=out)
    got, ref = _check(gpu_ctx, job, small_lines, init=init)
    np.testing.assert_array_equal(got[:5000], init[:5000])
    np.testing.assert_array_equal(got[5000 + 17777:], init[5000 + 17777:])


def test_zero_frequency_and_zero_intensity_lines(gpu_ctx, small_lines):
    L = {k: v.copy() for k, v in small_lines.items()}
    L["nu"][0] = 0.0          # nu0 == 0 -> 1e-6 (OpenMPManager.cpp:392)
    L["aif"][10:20] = 0.0     # S == 0 lines are skipped
    for prec in (capi.FP64, capi.FP32):
        job = _make(L, prec, capi.VOIGT, 16, capi.CONV_REF_CPU, nu0=0.0, dnu=0.1, G=41000)
        _check(gpu_ctx, job, L)


def test_fp64_bitwise_across_launch_shapes(gpu_ctx, small_lines):
    """FP64 bins sum their lines in line order whatever the tile shape."""
    res = []
    for cfg in [(2, 4, 0), (4, 4, 0), (8, 4, 0), (2, 8, 0), (4, 8, 0), (8, 8, 1)]:
        job = _make(small_lines, capi.FP64, capi.VOIGT, 16, capi.CONV_PHYSICAL)
        gpu_ctx.run([job], cfg=cfg); gpu_ctx.check()
        res.append(job.out.cpu().numpy())
    for r in res[1:]:
        np.testing.assert_array_equal(r, res[0])


def test_fp32_launch_shapes_within_tolerance(gpu_ctx, small_lines):
    for cfg in [(2, 4, 0), (4, 4, 0), (8, 4, 0), (2, 8, 0), (4, 8, 0), (8, 8, 0)]:
        job = _make(small_lines, capi.FP32, capi.VOIGT, 16, capi.CONV_PHYSICAL)
        gpu_ctx.run([job], cfg=cfg); gpu_ctx.check()
        ref = H.oracle_of(job, small_lines)
        rel, band = H.fp32_errors(job.out.cpu().numpy(), ref)
        assert rel <= H.FP32_REL and band <= H.FP32_BAND


def test_deterministic_repeat(gpu_ctx, small_lines):
    a = _make(small_lines, capi.FP32, capi.VOIGT, 16, capi.CONV_PHYSICAL)
    gpu_ctx.run([a]); gpu_ctx.check()
    first = a.out.clone()
    for _ in range(3):
        gpu_ctx.run([a]); gpu_ctx.check()
        assert torch.equal(a.out, first)


def test_eval_count_matches_oracle(gpu_ctx, small_lines):
    from oracle import pyoracle as po
    jobs = [_make(small_lines, capi.FP32, capi.VOIGT, 16, conv) for conv in
            (capi.CONV_PHYSICAL, capi.CONV_REF_CPU)]
    jobs.append(_make(small_lines, capi.FP64, capi.DOPPLER, 16, capi.CONV_REF_CPU, start_idx=100,
                      n_points=20000))
    got = gpu_ctx.count_evals(jobs)
    want = [po.count_evals(H.host_job(j.c, small_lines)) for j in jobs]
    assert got == want


@pytest.mark.parametrize("T,P,dnu", [(100.0, 1e-5, 0.1), (300.0, 1e-3, 0.1), (100.0, 1e-5, 0.005),
                                     (3000.0, 100.0, 0.1)])
def test_fp32_narrow_and_broad_lines(gpu_ctx, small_lines, T, P, dnu):
    """Lines far narrower than a bin (the nearest bins sit in the steep
    Doppler core) and pressure-broadened lines wider than many bins."""
    G = int(round(3900.0 / dnu)) + 1
    for prof in (capi.VOIGT, capi.DOPPLER):
        job = _make(small_lines, capi.FP32, prof, 16, capi.CONV_PHYSICAL, T=T, P=P, dnu=dnu, G=G,
                    cutoff=25.0)
        _check(gpu_ctx, job, small_lines)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("profile", [capi.VOIGT, capi.DOPPLER])
def test_prep_and_on_load_paths_agree_bitwise(gpu_ctx, small_lines, prec, profile):
    """Per-job prep of S(T), width and y (default) and derive-on-load give
    the same doubles, so the results are identical."""
    a = _make(small_lines, prec, profile, 16, capi.CONV_PHYSICAL, T=800.0, P=0.2)
    b = _make(small_lines, prec, profile, 16, capi.CONV_PHYSICAL, T=800.0, P=0.2)
    gpu_ctx.run([a], cfg=(4, 8, 0, 0))
    gpu_ctx.run([b], cfg=(4, 8, 0, capi.LAUNCH_DERIVE_ON_LOAD))
    gpu_ctx.check()
    assert torch.equal(a.out, b.out)


@pytest.mark.parametrize("nodes", [16, 32])
@pytest.mark.parametrize("P", [1e-3, 1.0, 100.0])
def test_gauss_hermite_fp32_across_pressures(gpu_ctx, small_lines, nodes, P):
    """FP32 Gauss-Hermite against the FP64 oracle of the same quadrature
    from narrow (y << 1, float-pair x near the nodes) to broad lines."""
    job = _make(small_lines, capi.FP32, capi.VOIGT_QUAD, nodes, capi.CONV_PHYSICAL, T=2500.0,
                P=P, nu0=1000.0, dnu=0.01, G=150000, cutoff=25.0)
    _check(gpu_ctx, job, small_lines)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("name,profile,nodes", [("voigt", capi.VOIGT, 16),
                                                ("doppler", capi.DOPPLER, 16),
                                                ("gh16", capi.VOIGT_QUAD, 16)])
def test_compact_line_list(gpu_ctx, small_lines, name, profile, nodes, prec):
    """GEXS_LINES_COMPACT (FP64 nu, float E'', g'A, gamma, n): the kernels
    compute on the widened floats, so the results match the oracle given
    those same values (g' = 1) with the usual tolerances; derive-on-load
    rejects the format."""
    cl = LineList(small_lines["nu"], small_lines["elow"], small_lines["aif"], small_lines["gns"],
                  small_lines["gamma"], small_lines["n"], compact=True)
    assert cl.elow.dtype == torch.float32 and cl.gns is None
    job = _make(small_lines, prec, profile, nodes, capi.CONV_PHYSICAL, lines_dev=cl)
    _check(gpu_ctx, job, cl.widened())
    bad = _make(small_lines, prec, profile, nodes, capi.CONV_PHYSICAL, lines_dev=cl)
    with pytest.raises(capi.GexsError):
        gpu_ctx.run([bad], cfg=(4, 8, 0, capi.LAUNCH_DERIVE_ON_LOAD))
