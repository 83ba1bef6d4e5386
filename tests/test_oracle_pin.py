"""Pin the FP64 oracle to the reference's own CPU code (no GPU needed).

Golden vectors come from tests/golden/make_golden.py, which runs the
reference's CPU path compiled from its sources.  The oracle must reproduce
them in the GEXS_CONV_REF_CPU convention:
  - Q(T), humlic: exactly (same arithmetic, same compiler semantics);
  - Voigt per bin: relative 1e-12 (observed ~1e-15: glibc exp/pow vs the
    same calls, only operand order in S(T) differs);
  - Doppler per bin: absolute 1e-12 of the peak.
"""
import os

import numpy as np
import pytest

from gexs_b200 import _capi as capi
from gexs_b200.engine import job_init
from oracle import pyoracle as po
from tests.helpers import host_job

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cpu.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _lines(g, tag):
    p = "lines_%s_" % tag
    return {k[len(p):]: v for k, v in g.items() if k.startswith(p)}


def test_partition_matches_reference(gold):
    for t, q in zip(gold["q_temps"], gold["q_ref"]):
        assert po.partition(gold["states_energy"], gold["states_g"], t) == q


def test_humlicek_matches_reference(gold):
    got = np.array([po.humlicek(x, y) for x, y in zip(gold["hum_x"], gold["hum_y"])])
    np.testing.assert_array_equal(got, gold["hum_ref"])


def test_humlicek_regions_all_covered(gold):
    regs = {po.orc().orc_humlicek_region(x, y) for x, y in zip(gold["hum_x"], gold["hum_y"])}
    assert regs == {1, 2, 3, 4}


def _voigt_job(gold, tag, i):
    nu0, dnu, n = gold["grid"]
    T, P = gold["voigt_cases"][i]
    q = float(gold["voigt_%s_%d_q" % (tag, i)][0])
    j = job_init(capi.CONV_REF_CPU, capi.VOIGT, T, P, q, 18.0, nu0, dnu, int(n), ref_temp=256.0)
    return j


@pytest.mark.parametrize("tag", ["wide", "narrow"])
@pytest.mark.parametrize("i", [0, 1, 2])
def test_voigt_matches_reference(gold, tag, i):
    L = _lines(gold, tag)
    hj = host_job(_voigt_job(gold, tag, i), L)
    got = po.cross_section(hj)
    ref = gold["voigt_%s_%d" % (tag, i)]
    assert np.array_equal(got == 0, ref == 0)
    m = ref != 0
    assert np.max(np.abs(got[m] - ref[m]) / np.abs(ref[m])) < 1e-12


def test_narrow_case_reaches_every_region(gold):
    L = _lines(gold, "narrow")
    hist = po.region_hist(host_job(_voigt_job(gold, "narrow", 1), L))
    assert all(h > 0 for h in hist), hist


@pytest.mark.parametrize("i", [0, 1])
def test_doppler_matches_reference(gold, i):
    L = _lines(gold, "wide")
    nu0, dnu, n = gold["grid"]
    T = float(gold["doppler_t"][i])
    q = float(gold["doppler_%d_q" % i][0])
    j = job_init(capi.CONV_REF_CPU, capi.DOPPLER, T, 1.0, q, 18.0, nu0, dnu, int(n))
    got = po.cross_section(host_job(j, L))
    ref = gold["doppler_%d" % i]
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(ref)


def test_stable_erf_form_agrees_with_literal(gold):
    """The cancellation-free erfc form differs from erf(xp)-erf(xm) only by
    the literal form's far-wing rounding noise (< 1e-14 of the peak)."""
    L = _lines(gold, "wide")
    nu0, dnu, n = gold["grid"]
    j = job_init(capi.CONV_REF_CPU, capi.DOPPLER, 1500.0, 1.0, 1000.0, 18.0, nu0, dnu, int(n))
    a = po.cross_section(host_job(j, L))
    j.erf_form = capi.ERF_STABLE
    b = po.cross_section(host_job(j, L))
    assert np.max(np.abs(a - b)) <= 1e-14 * np.max(a)


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
def test_live_reference_random_case(small_states):
    from gexs_b200 import synth
    L = synth.make_lines(small_states, 1500, 200.0, 900.0, 777, broadening_seed=778)
    L["gamma"] *= 0.05
    nu0, dnu, n = 150.0, 0.02, 40000
    freq = nu0 + np.arange(n, dtype=np.float64) * dnu
    T, P = 2200.0, 0.7
    q = po.ref_partition(small_states.energy, small_states.g, T)
    ref = po.ref_voigt_tp(freq, L, T, P, q, 28.0, 296.0, dnu, nthreads=3)
    j = job_init(capi.CONV_REF_CPU, capi.VOIGT, T, P, q, 28.0, nu0, dnu, n, ref_temp=296.0)
    got = po.cross_section(host_job(j, L))
    m = ref != 0
    assert np.array_equal(got == 0, ref == 0)
    assert np.max(np.abs(got[m] - ref[m]) / ref[m]) < 1e-12


def _header_list(name):
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "gexs_b200", "csrc", "gh_nodes.h")
    txt = open(path).read()
    body = re.search(r"#define %s \\\n(.*?)\n(?!    )" % name, txt, re.S).group(1)
    return np.array([float(v) for v in body.replace("\\", "").replace(",", " ").split()])


def test_gh_nodes_match_numpy_hermgauss():
    for nodes in (16, 32):
        t, w = np.polynomial.hermite.hermgauss(nodes)
        tp = _header_list("GEXS_GH%d_T_LIST" % nodes)
        wp = _header_list("GEXS_GH%d_W_LIST" % nodes)
        assert len(tp) == nodes // 2
        np.testing.assert_allclose(tp, t[t > 0], rtol=1e-13)
        np.testing.assert_allclose(wp, w[t > 0], rtol=1e-11)


def test_humlicek_against_faddeeva():
    """Humlicek W4's own accuracy against scipy's Faddeeva function: the
    approximation, not a parity target (~1e-4 relative)."""
    from scipy.special import wofz
    xs = np.linspace(0.0, 30.0, 301)
    worst = 0.0
    for y in (1e-4, 1e-2, 0.3, 1.0, 3.0, 10.0):
        k = np.array([po.humlicek(x, y) for x in xs])
        ref = wofz(xs + 1j * y).real
        worst = max(worst, float(np.max(np.abs(k - ref) / ref)))
    assert worst < 2e-4


def test_gh_converges_to_voigt_for_broad_lines():
    from scipy.special import wofz
    xs = np.linspace(0.0, 10.0, 101)
    for y in (2.0, 5.0):
        ref = wofz(xs + 1j * y).real
        k32 = np.array([po.voigt_gh(x, y, 32) for x in xs])
        assert np.max(np.abs(k32 - ref) / ref) < 1e-4
