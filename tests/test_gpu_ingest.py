"""GPU ExoMol ingest (gexs_exomol_*, gexs_b200/csrc/gexs_ingest.cu) against
the CPU restatement of the reference reader (oracle/ingest_oracle.cpp, pinned
to the reference in test_ingest_pin.py): bit-exact arrays, in file order and
sorted by nu, both broadening rules, the edge cases of the text format, and
the decimal parser against correctly rounded conversion."""
import os

import numpy as np
import pytest
import torch

from gexs_b200 import Job, LineList, synth, _capi as capi
from gexs_b200.engine import load_exomol, parse_exomol
from gexs_b200._capi import GexsError
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _text(nst=3000, ntr=20000, seed=61, nu_col=False):
    st = synth.make_states(nst, 40, seed)
    u, l, a = synth.make_exomol_transitions(st, ntr, 20.0, 8000.0, seed + 1)
    return st, synth.exomol_states_text(st), synth.exomol_trans_text(
        u, l, a, nu=(st.energy[u] - st.energy[l]) if nu_col else None)


def _bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.dtype == np.float64:
        return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))
    return np.array_equal(a, b)


def _cmp(got, ref):
    for k in ("nu", "elow", "aif", "gns", "gamma", "n"):
        g = got[k].cpu().numpy()
        assert _bits_equal(g, ref[k]), k


@pytest.mark.parametrize("sort", [False, True])
@pytest.mark.parametrize("mode", [capi.BROAD_DEFAULTS, capi.BROAD_BY_J])
def test_ingest_matches_oracle(gpu_ctx, sort, mode):
    st, stext, ttext = _text()
    broad = synth.exomol_broad_text(40, 9, a1_pairs=20)
    S, L = parse_exomol(gpu_ctx, stext, ttext, broad, mode, 0.07, 0.5, sort_by_nu=sort)
    e, g, j = po.exomol_states(stext)
    assert _bits_equal(S["energy"].cpu().numpy(), e)
    assert _bits_equal(S["g"].cpu().numpy(), g) and _bits_equal(S["J"].cpu().numpy(), j)
    ref = po.exomol_trans(ttext, e, g, j, broad, mode, 0.07, 0.5, sort_by_nu=sort)
    assert len(ref["nu"]) > 0
    _cmp(L, ref)
    if sort:
        nu = L["nu"].cpu().numpy()
        assert (np.diff(nu) >= 0).all()


def test_decimal_parser_is_correctly_rounded(gpu_ctx):
    """A column in many formats against Python's float() (correctly rounded,
    like glibc strtod)."""
    rng = np.random.Generator(np.random.PCG64(71))
    vals = []
    mags = 10.0 ** rng.uniform(-300, 300, 40000)
    for i, v in enumerate(mags):
        p = int(rng.integers(0, 17))
        vals.append(("%." + str(p) + "e") % v)
    for v in 10.0 ** rng.uniform(-8, 12, 20000):
        vals.append(("%." + str(int(rng.integers(0, 12))) + "f") % v)
    for _ in range(20000):                         # 15-19 significant digits
        nd = int(rng.integers(15, 20))
        digits = "".join(str(int(d)) for d in rng.integers(0, 10, nd))
        digits = str(int(rng.integers(1, 10))) + digits[1:]
        e = int(rng.integers(-30, 30))
        vals.append(digits[0] + "." + digits[1:] + "E" + ("%+d" % e))
    vals += ["0", "0.0", "-0.0", "1", "-1.5", "007", "1e22", "1e23", "9007199254740993",
             "4.9406564584124654e-300", "1.7976931348623157e+308", "2.2250738585072014e-307",
             "123456789012345678", "0.000000000000000000000012345", "+3.25E+02", ".5", "5."]
    text = "".join("1 1 %s\n" % v for v in vals).encode()
    stext = b"1 0.0 1 0\n"
    _, L = parse_exomol(gpu_ctx, stext, text, sort_by_nu=False)
    got = L["aif"].cpu().numpy()
    want = np.array([float(v) for v in vals])
    bad = np.nonzero(got.view(np.int64) != want.view(np.int64))[0]
    assert len(bad) == 0, [(vals[i], got[i], want[i]) for i in bad[:10]]


def test_text_edge_cases(gpu_ctx):
    """CRLF, no final newline, blank lines, a fourth column (ignored here:
    the reference's token stream would misread it, so the oracle gets the
    three-column text), octal-looking states fields."""
    st, stext, ttext = _text(nst=800, ntr=3000, seed=67)
    _, _, t4 = _text(nst=800, ntr=3000, seed=67, nu_col=True)
    s_lines = stext.rstrip(b"\n").split(b"\n")
    s2 = b"\r\n".join(ln if i % 5 else ln.replace(b"  " + str(int(st.g[i])).encode() + b" ",
                                                    b" 0" + str(int(st.g[i])).encode() + b" ", 1)
                      for i, ln in enumerate(s_lines))
    tl = ttext.split(b"\n")
    t2 = b"\n\n".join(tl[:100]) + b"\n" + b"\r\n".join(tl[100:]).rstrip(b"\r\n")
    S, L = parse_exomol(gpu_ctx, s2, t2, sort_by_nu=False)
    e, g, j = po.exomol_states(s2)
    assert _bits_equal(S["g"].cpu().numpy(), g)
    ref = po.exomol_trans(t2, e, g, j)
    _cmp(L, ref)
    # four columns: same lines as the three-column text
    S4, L4 = parse_exomol(gpu_ctx, stext, t4, sort_by_nu=False)
    ref3 = po.exomol_trans(ttext, *po.exomol_states(stext))
    _cmp(L4, ref3)


def test_errors_and_empty(gpu_ctx):
    st, stext, ttext = _text(nst=100, ntr=200, seed=73)
    with pytest.raises(GexsError):                 # id beyond the states
        parse_exomol(gpu_ctx, stext, b"1 101 1.0e-3\n")
    with pytest.raises(GexsError):                 # fewer than three fields
        parse_exomol(gpu_ctx, stext, b"1 2\n")
    with pytest.raises(GexsError):                 # a states line the reference would split
        parse_exomol(gpu_ctx, b"1 " + b" " * 1100 + b"0.0 1 0\n", b"1 1 1.0\n")
    S, L = parse_exomol(gpu_ctx, stext, b"")
    assert L["nu"].numel() == 0
    S, L = parse_exomol(gpu_ctx, stext, b"\n  \n")
    assert L["nu"].numel() == 0


def test_load_files_then_cross_section(gpu_ctx, tmp_path):
    """gexs_exomol_load from files, then an FP64 Voigt cross-section of the
    ingested list against the oracle on the same (oracle-parsed) lines."""
    st, stext, ttext = _text(nst=2000, ntr=6000, seed=79)
    broad = synth.exomol_broad_text(40, 11)
    paths = []
    for name, data in (("x.states", stext), ("x.trans", ttext), ("x.broad", broad)):
        p = os.path.join(str(tmp_path), name)
        with open(p, "wb") as f:
            f.write(data)
        paths.append(p)
    S, L = load_exomol(gpu_ctx, paths[0], paths[1], paths[2], capi.BROAD_BY_J, 0.07, 0.5)
    e, g, j = po.exomol_states(stext)
    ref = po.exomol_trans(ttext, e, g, j, broad, capi.BROAD_BY_J, 0.07, 0.5, sort_by_nu=True)
    _cmp(L, ref)
    # missing broadener file: defaults
    _, Ld = load_exomol(gpu_ctx, paths[0], paths[1], paths[2] + ".missing", capi.BROAD_BY_J, 0.07, 0.5)
    assert (Ld["gamma"] == 0.07).all() and (Ld["n"] == 0.5).all()
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"])
    q = po.partition(e, g, 1200.0)
    G = 20000
    out = torch.zeros(G, dtype=torch.float64, device="cuda")
    jb = Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=1200.0,
             pressure=1.0, partition=q, mass=18.0, nu_start=100.0, dnu=0.4, grid_points=G,
             precision=capi.FP64, cutoff=25.0)
    gpu_ctx.run([jb])
    gpu_ctx.check()
    host = {"nu": ref["nu"], "elow": ref["elow"], "aif": ref["aif"], "gns": ref["gns"],
            "gamma": ref["gamma"], "n": ref["n"]}
    want = po.cross_section(H.host_job(jb.c, host))
    worst, nbad = H.fp64_mismatch(out.cpu().numpy(), want)
    assert nbad == 0, worst


@pytest.mark.parametrize("sort", [False, True])
def test_hitran_matches_oracle(gpu_ctx, sort):
    """gexs_hitran_parse against the restated HITRANStateReader (pinned to
    the reference in test_ingest_pin.py): nu, E'', gamma, n, g' bit-exact, A
    bit-exact where the file gives it; where it is rebuilt from S the GPU's
    FP64 exp stands in for glibc's: within 4 ulp."""
    from gexs_b200.engine import parse_hitran
    text = synth.make_hitran_par(30000, 89)
    got = parse_hitran(gpu_ctx, text, pressure=0.8, air_mixture=0.7, ref_partition_296=174.58,
                       sort_by_nu=sort)
    ref = po.hitran(text, 0.8, 0.7, 174.58, sort_by_nu=sort)
    for k in ("nu", "elow", "gamma", "n", "gns"):
        assert _bits_equal(got[k].cpu().numpy(), ref[k]), k
    a, b = got["aif"].cpu().numpy(), ref["aif"]
    rebuilt = ref["gns"] == 1
    assert _bits_equal(a[~rebuilt], b[~rebuilt])
    ulp = np.spacing(np.abs(b[rebuilt]))
    assert (np.abs(a[rebuilt] - b[rebuilt]) <= 4 * ulp).all()


def test_hitran_cross_section_at_1000_K_with_tips(gpu_ctx):
    """The synthetic .par file is H2O 161 (molecule 1, isotopologue 1).
    ref_partition_296 = 0 makes gexs_hitran_parse take Q(296) for the A it
    rebuilds from S from TIPS-2011, as the reference does
    (HITRANStateReader.cpp:88-95); Q(1000 K) for S(T) comes from
    gexs_tips_2011 too (:128).  Lines against the oracle's parse with the
    same Q(296) (A rebuilt within 4 ulp), then the FP64 Voigt cross-section
    at 1000 K against the FP64 oracle within 1e-10 per bin."""
    import ctypes as C
    from gexs_b200.engine import parse_hitran
    gi, q296, q1000 = C.c_double(), C.c_double(), C.c_double()
    capi.check(capi.lib().gexs_tips_2011(1, 1, 296.0, C.byref(gi), C.byref(q296)), "tips")
    capi.check(capi.lib().gexs_tips_2011(1, 1, 1000.0, C.byref(gi), C.byref(q1000)), "tips")
    assert 170.0 < q296.value < 180.0 and q1000.value > q296.value
    text = synth.make_hitran_par(20000, 93)
    got = parse_hitran(gpu_ctx, text, pressure=1.0, air_mixture=0.7, ref_partition_296=0.0,
                       sort_by_nu=True)
    ref = po.hitran(text, 1.0, 0.7, q296.value, sort_by_nu=True)
    a, b = got["aif"].cpu().numpy(), ref["aif"]
    assert (np.abs(a - b) <= 4 * np.spacing(np.abs(b))).all()
    lines = LineList(got["nu"], got["elow"], got["aif"], got["gns"], got["gamma"], got["n"])
    host = {k: got[k].cpu().numpy() for k in ("nu", "elow", "aif", "gns", "gamma", "n")}
    G = 300000
    out = torch.zeros(G, dtype=torch.float64, device="cuda")
    j = Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=1000.0,
            pressure=1.0, partition=q1000.value, mass=18.0, nu_start=500.0, dnu=0.025,
            grid_points=G, precision=capi.FP64, cutoff=25.0)
    gpu_ctx.run([j])
    gpu_ctx.check()
    want = H.oracle_of(j, host)
    assert want.max() > 0
    worst, nbad = H.fp64_mismatch(out.cpu().numpy(), want)
    assert nbad == 0, worst
